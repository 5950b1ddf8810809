"""Chained execution: a state of at most 32 MiB runs every pass of its plan in
one persistent launch (kernels.cu chain_kernel), each pass's tiles waiting
(bounded) for the tiles of the passes before it.  The chained run must give
the per-pass launches' result -- bit for bit in FP64, where both apply the same
tile code in the same order -- and the oracle's, with one kernel launch.
"""
import numpy as np
import pytest

from simulador_quantico_b200 import workloads as wl
from tests.helpers import TOL_F32, TOL_F64, oracle_state, random_gate_circuit_spec, random_state

pytestmark = pytest.mark.gpu


def run(sq, spec, prec, init, chained, iterations=1, **kw):
    c = spec.build(sq.Circuit())
    plan = sq.Plan(c, spec.qubits, prec, chained=chained, **kw)
    st = sq.State(spec.qubits, prec).upload(init)
    plan.upload()
    sq.synchronize()
    l0 = sq.kernel_launches()
    st.execute(plan, iterations)
    launches = sq.kernel_launches() - l0
    plan.status()
    out = st.download()
    st.free()
    return out, launches, plan.stats()["passes"]


@pytest.mark.parametrize("n,prec,reg_bits", [(13, "f64", -1), (15, "f64", -1), (21, "f64", -1), (14, "f32", -1),
                                              (18, "f32", -1), (22, "f32", -1), (13, "f32", 4), (20, "f32", 4)])
def test_chained_equals_per_pass(sq, n, prec, reg_bits):
    spec = random_gate_circuit_spec(n, 8 * n, seed=500 + n)
    init = random_state(n, seed=n, dtype=np.complex128 if prec == "f64" else np.complex64)
    a, la, passes = run(sq, spec, prec, init, 1, renorm_every=0, reg_bits=reg_bits)
    b, lb, _ = run(sq, spec, prec, init, 0, renorm_every=0, reg_bits=reg_bits)
    assert passes >= 2
    assert la == 1 and lb == passes
    assert np.array_equal(a, b)
    want = oracle_state(spec, "f64", init=init)
    assert np.abs(a - want).max() < (TOL_F64 if prec == "f64" else TOL_F32)


def test_chained_iterations_and_renorm(sq):
    """An FP32 Grover search of 16 qubits, every pass and the renormalisation
    every 64 passes in one launch, over 4 runs of a one-iteration plan too."""
    n, w = 16, 12345
    spec = wl.grover_search(n, w)
    init = np.zeros(1 << n, dtype=np.complex64)
    init[0] = 1
    got, launches, passes = run(sq, spec, "f32", init, 1)
    assert launches == 1 and passes > 64
    want = oracle_state(spec, "f64")
    assert np.abs(got - want).max() < 1e-4
    # renormalised every 64 passes: FP32 drift of at most 63 passes remains
    assert abs(np.vdot(got.astype(np.complex128), got.astype(np.complex128)).real - 1.0) < 1e-4
    assert int(np.argmax(np.abs(got))) == w
    # a one-iteration plan run 4 times: the chained sequence spans the iterations
    it_spec = wl.grover_search(n, w, iterations=4)
    (h_steps, _, _), (it_steps, _, _) = it_spec.calls
    one = wl.CircuitSpec("one", n, 0, it_spec.gates, [(it_steps, 1, True)])
    start = oracle_state(wl.CircuitSpec("h", n, 0, {}, [([h_steps[0]], 1, True)]), "f64")
    got4, l4, _ = run(sq, one, "f64", start, 1, iterations=4)
    assert l4 == 1
    assert np.abs(got4 - oracle_state(it_spec, "f64")).max() < TOL_F64


def test_chained_many_iterations_fp32_renorm(sq):
    """A one-iteration FP32 Grover plan run 300 times: 600 passes and 9
    renormalisations in one launch, through the chained kernel's three norm
    slots used in turn; the result matches the per-pass launches and the
    oracle, and stays normalised."""
    n, w, k = 15, 4321, 300
    it_spec = wl.grover_search(n, w, iterations=k)
    (h_steps, _, _), (it_steps, _, _) = it_spec.calls
    one = wl.CircuitSpec("one", n, 0, it_spec.gates, [(it_steps, 1, True)])
    start = oracle_state(wl.CircuitSpec("h", n, 0, {}, [([h_steps[0]], 1, True)]), "f64").astype(np.complex64)
    a, la, passes = run(sq, one, "f32", start, 1, iterations=k)
    b, lb, _ = run(sq, one, "f32", start, 0, iterations=k)
    assert la == 1 and lb == passes * k and passes * k > 9 * 64
    assert np.abs(a - b).max() < 1e-5
    want = oracle_state(it_spec, "f64")
    assert np.abs(a - want).max() < 1e-4
    assert abs(np.vdot(a.astype(np.complex128), a.astype(np.complex128)).real - 1.0) < 1e-4
