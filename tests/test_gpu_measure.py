"""Device-resident measurement against the reference's own DGM.

hgm_measure_qubit restates DGM::measure(int) (src/core/dgm_core.cpp:69-125):
outcome 0 iff P(0) > the uniform sample, then the measured branch,
renormalised, is moved to the qubit's |0> half and the |1> half cleared.
hgm_collapse_qubit restates DGM::colapse (dgm_core.cpp:129-146) and
hgm_marginal_probs DGM::measure(vector<int>) (dgm_core.cpp:150-162).

Each case runs the reference's DGM (oracle/_ref/libref_{f64,f32}.so, built
from the reference sources) and the engine on the same state.  The sample
the reference draws from its generator after seed_rng(seed) is handed to the
engine, so both take the same outcome.  FP64 states must agree within 1e-12;
FP32 states within 2e-5 (the reference accumulates its sums in float).
"""
import numpy as np
import pytest

from oracle import cpu
from simulador_quantico_b200 import workloads as wl
from tests.helpers import TOL_F32, TOL_F64, engine_state, random_state

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (cpu.ref_available("f64") and cpu.ref_available("f32")),
                                 reason="reference engine not built")]

TOL = {"f64": TOL_F64, "f32": TOL_F32}
DT = {"f64": np.complex128, "f32": np.complex64}


def ref_dgm(n, prec, init):
    r = cpu.RefDGM(n, prec)
    r.set_state(init)
    return r


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [3, 11, 16])
def test_measure_qubit_matches_reference(sq, prec, n):
    rng = np.random.default_rng(100 + n)
    init = random_state(n, seed=n, dtype=DT[prec])
    outcomes = set()
    for trial in range(6):
        q = int(rng.integers(n))
        seed = int(rng.integers(1 << 31))
        r = ref_dgm(n, prec, init)
        sample = r.uniform_sample(seed)
        bit = n - 1 - q
        p0 = float(np.sum(np.abs(init[((np.arange(1 << n) >> bit) & 1) == 0].astype(np.complex128)) ** 2))
        if abs(p0 - sample) < 1e-5:
            r.close()
            continue  # too close to call in FP32
        want_out = r.measure(q)
        want = r.state()
        r.close()
        st = sq.State(n, prec).upload(init)
        got_out, p = st.measure_qubit(q, sample)
        got = st.download()
        st.free()
        assert got_out == want_out, (trial, q, sample, p0)
        assert abs(p - (1 - p0 if got_out else p0)) < 1e-6
        assert np.abs(got - want).max() < TOL[prec], (trial, q)
        # the qubit is left in |0> whichever value was read
        assert np.all(got[((np.arange(1 << n) >> bit) & 1) == 1] == 0)
        outcomes.add(got_out)
    assert outcomes == {0, 1}


def test_measure_sequence_after_grover(sq):
    """grover.out's read-out (src/algorithms/lib_grover.cpp:61-63): after the
    search, measure qubits 1..n-1 in turn, each with the reference's next
    sample; outcomes and the final state agree with the reference's DGM."""
    n, w = 12, 1234
    spec = wl.grover_reference(n, w)
    init_state, _ = engine_state(sq, spec, "f64")
    r = ref_dgm(n, "f64", init_state)
    st = sq.State(n, "f64").upload(init_state)
    for q in range(1, n):
        sample = r.uniform_sample(7000 + q)
        assert st.measure_qubit(q, sample)[0] == r.measure(q)
    assert np.abs(st.download() - r.state()).max() < TOL_F64
    st.free()
    r.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_collapse_matches_reference(sq, prec):
    n = 14
    init = random_state(n, seed=5, dtype=DT[prec])
    for q, v in [(0, 0), (3, 1), (13, 1), (7, 0)]:
        r = ref_dgm(n, prec, init)
        r.colapse(q, v)
        want = r.state()
        r.close()
        st = sq.State(n, prec).upload(init)
        p = st.collapse_qubit(q, v)
        got = st.download()
        st.free()
        bit = n - 1 - q
        sel = ((np.arange(1 << n) >> bit) & 1) == v
        assert abs(p - np.sum(np.abs(init[sel].astype(np.complex128)) ** 2)) < 1e-6
        assert np.abs(got - want).max() < TOL[prec], (q, v)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("qubits", [[0], [2, 5], [1, 4, 9, 12], list(range(0, 14, 2)), list(range(1, 13))])
def test_measure_positions_matches_reference(sq, prec, qubits):
    """DGM::measure(vector<int>): every value's probability, keyed by index & mask."""
    n = 14
    init = random_state(n, seed=9, dtype=DT[prec])
    r = ref_dgm(n, prec, init)
    want = r.measure_many(qubits)
    r.close()
    dgm = sq.DGM(qubits=n, precision=prec)
    dgm.allocateMemory()
    dgm.state.upload(init)
    got = dgm.measure_positions(qubits)
    assert set(got) == set(want)
    tol = 1e-12 if prec == "f64" else 1e-5
    for k in want:
        assert abs(got[k] - want[k]) < tol, (k, got[k], want[k])
    assert abs(sum(got.values()) - 1.0) < 1e-6


def test_marginal_probs_large_mask(sq):
    """A mask of more values than the chunked path takes (2^12 > 1184), against numpy."""
    n = 16
    init = random_state(n, seed=3)
    st = sq.State(n, "f64").upload(init)
    mask = 0b1010110101101011
    got = st.marginal_probs(mask)
    st.free()
    bits = [b for b in range(n) if (mask >> b) & 1]
    idx = np.arange(1 << n)
    x = np.zeros(1 << n, dtype=np.int64)
    for j, b in enumerate(bits):
        x |= ((idx >> b) & 1) << j
    want = np.bincount(x, weights=np.abs(init) ** 2, minlength=1 << len(bits))
    assert np.abs(got - want).max() < 1e-14
