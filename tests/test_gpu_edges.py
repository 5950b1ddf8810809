"""Edge cases on the GPU: empty circuits, the smallest states, the sizes
where the engine switches path (shared-memory state, one tile, two tiles),
iterations = 0, refused inputs, both marginal-argmax paths, and the largest
states (32 qubits FP32 and 33 qubits FP64, checked through size-independent
properties: the norm, bit probabilities and the marginal argmax).
"""
import math

import numpy as np
import pytest

from tests.helpers import TOL_F32, TOL_F64, engine_state, oracle_state, random_gate_circuit_spec, random_state

pytestmark = pytest.mark.gpu

TOL = {"f64": TOL_F64, "f32": TOL_F32}
H = np.array([1, 1, 1, -1]) / math.sqrt(2)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_empty_circuit_leaves_state(sq, prec):
    n = 12
    init = random_state(n, seed=5)
    st = sq.State(n, prec).upload(init)
    st.execute(sq.Plan(sq.Circuit(), n, prec))
    got = st.download()
    st.free()
    assert np.abs(got - init.astype(got.dtype)).max() == 0.0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_empty_pt_list_through_wrapper(sq, prec):
    """GpuExecutionWrapper with a PT list holding only its NULL terminator."""
    L = sq.load_dropin(prec)
    n = 10
    init = random_state(n, seed=6).astype(np.complex128 if prec == "f64" else np.complex64)
    host = init.copy()
    empty = sq.Circuit()  # owns the PT array: keep it alive across the call
    pts = empty.ref_pts(prec)
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, 1)
    assert np.array_equal(host, init)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [1, 2, 3])
def test_smallest_states(sq, prec, n):
    spec = random_gate_circuit_spec(n, 6 * n + 3, seed=100 + n, max_controls=n - 1)
    init = random_state(n, seed=n)
    got, _ = engine_state(sq, spec, prec, init=init)
    assert np.abs(got - oracle_state(spec, "f64", init=init)).max() < TOL[prec]


@pytest.mark.parametrize("prec,n", [("f64", 8), ("f64", 9), ("f64", 11), ("f64", 12),
                                    ("f32", 9), ("f32", 10), ("f32", 12), ("f32", 13)])
def test_path_boundaries(sq, prec, n):
    """Around the switch from the shared-memory path to register tiles
    (5+R qubits) and from one tile to two (5+R+W with W = 2)."""
    spec = random_gate_circuit_spec(n, 10 * n, seed=7 * n, max_controls=3)
    init = random_state(n, seed=n + 50)
    got, _ = engine_state(sq, spec, prec, init=init)
    assert np.abs(got - oracle_state(spec, "f64", init=init)).max() < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_zero_iterations(sq, prec):
    spec = random_gate_circuit_spec(14, 40, seed=3)
    init = random_state(14, seed=4)
    got, _ = engine_state(sq, spec, prec, init=init, iterations=0)
    assert np.array_equal(got, init.astype(got.dtype))


def test_refused_inputs(sq):
    c = sq.Circuit()
    c.append_op(0, 0, 0, H)
    st = sq.State(10, "f64")
    with pytest.raises(sq.HgmError):
        st.set_basis(1 << 10)                       # index outside the state
    with pytest.raises(sq.HgmError):
        st.execute(sq.Plan(c, 11, "f64"))          # plan for another size
    with pytest.raises(sq.HgmError):
        st.execute(sq.Plan(c, 10, "f32"))          # plan of the other precision
    with pytest.raises(sq.HgmError):
        sq.State(35, "f32")                         # beyond the 34-qubit limit
    st.free()


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("bits", [(), (0,), (3, 7, 12), tuple(range(1, 11)), tuple(range(11)), tuple(range(14))])
def test_marginal_argmax_paths(sq, prec, bits):
    """Both marginal paths (chunked, for masks of up to 1184 values; one
    thread per value above that) against the marginal computed on the host
    from the same state."""
    n = 14
    rng = np.random.default_rng(len(bits) + 3)
    amp = rng.normal(size=1 << n) * np.exp(rng.uniform(0, 6.3, 1 << n) * 1j)
    amp /= np.linalg.norm(amp)
    st = sq.State(n, prec).upload(amp)
    host = st.download().astype(np.complex128)
    mask = 0
    for b in bits:
        mask |= 1 << b
    idx, p = st.marginal_argmax(mask)
    st.free()
    probs = np.abs(host) ** 2
    x = np.zeros(1 << n, dtype=np.int64)
    for k, b in enumerate(bits):
        x |= ((np.arange(1 << n) >> b) & 1) << k
    marg = np.bincount(x, weights=probs, minlength=1 << len(bits))
    want = int(np.argmax(marg))
    assert abs(p - marg[want]) < 1e-12
    assert idx == want or abs(marg[idx] - marg[want]) < 1e-15


@pytest.mark.parametrize("prec,n", [("f32", 32), ("f64", 33)])
def test_largest_states(sq, prec, n):
    """64-bit index arithmetic at 32 / 33 qubits: H on the lowest and the
    highest index bit, a phase, and an X on bit 5 controlled by the highest
    bit; checked by norm, bit probabilities and a two-bit marginal argmax."""
    free, _ = sq.mem_info()
    need = (8 if prec == "f32" else 16) << n
    if free < need + (4 << 30):
        pytest.skip(f"needs {need / 2**30:.0f} GiB free on the device")
    c = sq.Circuit()
    c.append_op(n - 1, 0, 0, H)
    c.append_op(0, 0, 0, H)
    c.append_op(0, 0, 0, [1, 0, 0, np.exp(0.7j)])
    c.append_op(5, 1 << (n - 1), 1 << (n - 1), [0, 1, 1, 0])
    st = sq.State(n, prec).set_basis(0)
    st.execute(sq.Plan(c, n, prec))
    assert abs(st.norm() - 1.0) < 1e-6
    assert abs(st.prob_one(n - 1) - 0.5) < 1e-6
    assert abs(st.prob_one(0) - 0.5) < 1e-6
    assert abs(st.prob_one(5) - 0.5) < 1e-6                # follows bit n-1
    idx, p = st.marginal_argmax((1 << 5) | 1)
    assert abs(p - 0.25) < 1e-6 and idx in (0, 1, 2, 3)
    st.free()


@pytest.mark.parametrize("prec,n", [("f32", 25), ("f64", 26), ("f32", 28)])
def test_staged_copy_round_trip(sq, prec, n):
    """States of 256 MiB and more travel through page-locked staging chunks on
    several host threads.  A chunk placed at the wrong offset would change the
    per-bit probabilities the device computes; a byte lost on the way back
    would break the exact round trip."""
    rng = np.random.default_rng(n)
    dt = np.complex64 if prec == "f32" else np.complex128
    amp = np.empty(1 << n, dtype=dt)
    amp.real = rng.random(1 << n)
    amp.imag = np.arange(1 << n) / float(1 << n)     # index-dependent
    st = sq.State(n, prec).upload(amp)
    w = np.abs(amp.astype(np.complex128)) ** 2
    total = w.sum()
    assert abs(st.norm() - total) < 1e-6 * total
    idx = np.arange(1 << n, dtype=np.int64)
    for b in (0, 7, n - 5, n - 2, n - 1):
        want = w[(idx >> b) & 1 == 1].sum()              # prob_one is not normalised
        assert abs(st.prob_one(b) - want) < 1e-6 * total, b
    back = st.download()
    st.free()
    assert np.array_equal(back.view(np.uint8), amp.view(np.uint8))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_plan_freed_right_after_queueing(sq, prec):
    """A plan dropped as soon as the execution that uses it is queued (a
    temporary in Python) is freed only after the device finishes with it."""
    n = 20
    spec = random_gate_circuit_spec(n, 120, seed=3)
    init = random_state(n, seed=8)
    st = sq.State(n, prec).upload(init)
    for _ in range(3):
        st.execute(sq.Plan(spec.build(sq.Circuit()), n, prec))  # the plan is freed on return
    got = st.download()
    st.free()
    want = init
    for _ in range(3):
        want = oracle_state(spec, "f64", init=want)
    assert np.abs(got - want.astype(got.dtype)).max() < 10 * TOL[prec]
