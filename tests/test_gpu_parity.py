"""Engine vs oracle on the GPU: every result within the stated tolerance.

FP64: max |amplitude - oracle| <= 1e-12.  FP32: <= 2e-5 against the FP32
oracle and 1 - F < 1e-6 against the FP64 oracle.  The oracle is the C
restatement of the reference's serial CPU path (oracle/sv_oracle.c).
"""
import math

import numpy as np
import pytest

from oracle import closed_forms as cf
from oracle import circuit_lang as cl
from oracle import cpu
from simulador_quantico_b200 import workloads as wl
from tests.helpers import (TOL_F32, TOL_F64, engine_state, fidelity_gap, min_tiled_qubits, oracle_state,
                           random_gate_circuit_spec, random_state)

pytestmark = pytest.mark.gpu


# ---- the reference's own truth tables (tests/test_gates.cpp:43-90) ------------

GATE_CASES = [
    ("CNot", 2, lambda: cl.CNot(2, 0, 1, 1), lambda s: [0, 1, 3, 2][s]),
    ("Toffoli", 3, lambda: cl.Toffoli(3, 0, 1, 2, 3), lambda s: [0, 1, 2, 3, 4, 5, 7, 6][s]),
    ("ControlledN", 4, lambda: cl.ControlledN(4, [0, 1, 2], 3, "X", -1), lambda s: (s ^ 1) if (s >> 1) == 7 else s),
    ("Controlled1(ctrl=0)", 2, lambda: cl.Controlled1(2, 0, 1, "X", 0), lambda s: [1, 0, 2, 3][s]),
]


@pytest.mark.parametrize("name,n,circ,expected", GATE_CASES, ids=[c[0] for c in GATE_CASES])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_reference_truth_tables(sq, name, n, circ, expected, prec):
    for start in range(1 << n):
        rb = min(8, n)
        dgm = sq.DGM(qubits=n, precision=prec, gpu_region_bits=rb, gpu_coalesced_bits=min(4, rb),
                     block_size=1 << (rb - 2), repeat_count=2)
        dgm.allocateMemory()
        dgm.setMemoryValue(start)
        dgm.executeFunction(circ())
        got = dgm.host_state()
        want = np.zeros(1 << n)
        want[expected(start)] = 1.0
        assert np.abs(got - want).max() < 1e-6, (name, start)


@pytest.mark.parametrize("n", [10, 11, 12, 13, 14])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
def test_embedded_truth_tables(sq, n, warp_bits):
    """The same controlled-X truth tables on every placement inside an n-qubit register."""
    if min_tiled_qubits("f64", warp_bits) > n:
        pytest.skip("tile larger than state")
    rng = np.random.default_rng(n * 10 + warp_bits)
    for trial in range(6):
        qs = rng.choice(n, size=4, replace=False)
        steps = [cl.CNot(n, int(qs[0]), int(qs[1]), 1), cl.Toffoli(n, int(qs[1]), int(qs[2]), int(qs[3]), 2),
                 cl.ControlledN(n, [int(qs[3]), int(qs[0])], int(qs[2]), "X", 1)]
        spec = wl.CircuitSpec("ctrl", n, int(rng.integers(1 << n)), {}, [(steps, 1, True)])
        got, _ = engine_state(sq, spec, "f64", warp_bits=warp_bits)
        want = oracle_state(spec, "f64")
        assert np.array_equal(np.abs(got) > 0.5, np.abs(want) > 0.5)
        assert np.abs(got - want).max() < TOL_F64


@pytest.mark.parametrize("n", [3, 8, 9, 10, 11, 12, 13, 15])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
@pytest.mark.parametrize("fuse", [1, 0])
def test_random_gates_f64(sq, n, warp_bits, fuse):
    lo = min_tiled_qubits("f64")
    if n >= lo and lo + warp_bits > n:
        pytest.skip("tile larger than state")
    if n < lo and warp_bits:
        pytest.skip("small-state path has no warp bits")
    spec = random_gate_circuit_spec(n, 6 * n + 12, seed=n * 100 + warp_bits * 10 + fuse)
    init = random_state(n, seed=n)
    got, _ = engine_state(sq, spec, "f64", init=init, warp_bits=warp_bits, fuse=fuse)
    want = oracle_state(spec, "f64", init=init)
    assert np.abs(got - want).max() < TOL_F64


@pytest.mark.parametrize("low_bits", [0, 1, 3, 5])
def test_random_gates_low_bits(sq, low_bits):
    n = 16
    spec = random_gate_circuit_spec(n, 120, seed=low_bits + 7)
    init = random_state(n, seed=3)
    got, _ = engine_state(sq, spec, "f64", init=init, low_bits=low_bits)
    want = oracle_state(spec, "f64", init=init)
    assert np.abs(got - want).max() < TOL_F64


@pytest.mark.parametrize("n", [8, 10, 12, 16])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
def test_random_gates_f32(sq, n, warp_bits):
    lo = min_tiled_qubits("f32")
    if n >= lo and lo + warp_bits > n:
        pytest.skip("tile larger than state")
    if n < lo and warp_bits:
        pytest.skip("small-state path has no warp bits")
    spec = random_gate_circuit_spec(n, 5 * n, seed=n + warp_bits)
    init = random_state(n, seed=n + 1)
    got, _ = engine_state(sq, spec, "f32", init=init.astype(np.complex64), warp_bits=warp_bits, renorm_every=0)
    want32 = oracle_state(spec, "f32", init=init.astype(np.complex64))
    want64 = oracle_state(spec, "f64", init=init)
    assert np.abs(got - want32).max() < TOL_F32
    assert fidelity_gap(got, want64) < 1e-6


@pytest.mark.parametrize("n", [9, 12, 16])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
def test_random_gates_f32_sixteen_registers(sq, n, warp_bits):
    """FP32 tiles of 16 amplitudes a thread (reg_bits = 4)."""
    if 9 + warp_bits > n:
        pytest.skip("tile larger than state")
    spec = random_gate_circuit_spec(n, 5 * n, seed=n + warp_bits + 40)
    init = random_state(n, seed=n + 2)
    got, stats = engine_state(sq, spec, "f32", init=init.astype(np.complex64), warp_bits=warp_bits,
                              renorm_every=0, reg_bits=4)
    assert stats["reg_bits"] == 4
    assert np.abs(got - oracle_state(spec, "f32", init=init.astype(np.complex64))).max() < TOL_F32
    assert fidelity_gap(got, oracle_state(spec, "f64", init=init)) < 1e-6


@pytest.mark.parametrize("n,warp_bits", [(13, 0), (14, 2), (18, 3), (20, 2)])
def test_split_layers(sq, n, warp_bits):
    """Layers of Rz.Ry gates as phase, packed real gate, phase, with CNOTs
    that relabel register bits between them (the relabeled bits take the
    conjugated phases and the per-thread factor): FP32 and FP64 split plans
    against the FP64 oracle, and FP32 split against FP32 dense."""
    spec = wl.random_layered(n, 6, seed=n + 3)
    want = oracle_state(spec, "f64")
    got64, _ = engine_state(sq, spec, "f64", warp_bits=warp_bits, split_layers=1)
    assert np.abs(got64 - want).max() < TOL_F64
    split, _ = engine_state(sq, spec, "f32", warp_bits=warp_bits, split_layers=1, renorm_every=0)
    dense, _ = engine_state(sq, spec, "f32", warp_bits=warp_bits, split_layers=0, renorm_every=0)
    assert fidelity_gap(split, want) < 1e-6
    assert np.abs(split - want).max() < TOL_F32
    assert np.abs(split - dense).max() < TOL_F32


def zyz_layered(n, layers, seed):
    """Layers of Rz.Ry.Rz on every qubit (a phase on both sides of each split
    gate's real part) and CNOTs on a random matching."""
    rng = np.random.default_rng(seed)
    gates, steps = {}, []
    for layer in range(layers):
        for tag, fn in (("a", wl.rz), ("b", wl.ry), ("c", wl.rz)):
            names = []
            for q in range(n):
                name = f"{tag}{layer}_{q}"
                gates[name] = fn(float(rng.uniform(0.0, 2.0 * math.pi)))
                names.append(name)
            steps.append(",".join(names))
        perm = rng.permutation(n)
        row = ["ID"] * n
        for g in range(n // 2):
            row[int(perm[2 * g])] = f"Control{g + 1}(1)"
            row[int(perm[2 * g + 1])] = f"Target{g + 1}(X)"
        steps.append(",".join(row))
    return wl.CircuitSpec("zyz", n, 0, gates, [(steps, 1, True)])


@pytest.mark.parametrize("n,warp_bits", [(14, 2), (18, 3)])
def test_split_layers_post_phase(sq, n, warp_bits):
    """Split gates with a phase after the real part too (Rz.Ry.Rz; that phase
    follows the split layer as a phase record): FP32 against the FP64 oracle."""
    spec = zyz_layered(n, 4, seed=n)
    want = oracle_state(spec, "f64")
    got, _ = engine_state(sq, spec, "f32", warp_bits=warp_bits, renorm_every=0)
    assert np.abs(got - want).max() < TOL_F32
    assert fidelity_gap(got, want) < 1e-6


# ---- benchmark shapes at oracle-checkable sizes --------------------------------

def test_hadamard_benchmark_20q(sq):
    """general.out 20: every amplitude 2^-10 (config-1 shape, FP64, 1e-12)."""
    spec = wl.hadamard_benchmark(20, 3)
    got, stats = engine_state(sq, spec, "f64")
    assert np.abs(got - cf.hadamard_all(20)).max() < TOL_F64
    assert np.abs(got - oracle_state(spec)).max() < TOL_F64


@pytest.mark.parametrize("n", [11, 13])
def test_grover_reference_form(sq, n):
    w = 42 % (1 << (n - 1))
    spec = wl.grover_reference(n, w)
    got, _ = engine_state(sq, spec, "f64")
    want = oracle_state(spec)
    assert np.abs(got - want).max() < TOL_F64
    k = spec.meta["iterations"]
    assert np.abs(got - cf.grover_reference_form(n, w, k)).max() < 1e-11


def test_grover_search_argmax(sq):
    m, w = 14, 42
    spec = wl.grover_search(m, w)
    c = spec.build(sq.Circuit())
    st = sq.State(m, "f64").set_basis(0)
    st.execute(sq.Plan(c, m, "f64"))
    arg, p = st.marginal_argmax((1 << m) - 1)
    marked, _ = cf.grover_amplitudes(m, spec.meta["iterations"])
    assert arg == w
    assert abs(p - marked ** 2) < 1e-12
    want = cf.grover_search(m, w, spec.meta["iterations"])
    assert np.abs(st.download() - want).max() < 1e-11


@pytest.mark.parametrize("n,layers", [(12, 4), (16, 3), (18, 2)])
def test_random_layered(sq, n, layers):
    spec = wl.random_layered(n, layers, seed=n)
    got, _ = engine_state(sq, spec, "f64")
    assert np.abs(got - oracle_state(spec)).max() < TOL_F64
    got32, _ = engine_state(sq, spec, "f32")
    assert fidelity_gap(got32, got) < 1e-6


@pytest.mark.parametrize("n", [10, 12, 14])
def test_qft_closed_form(sq, n):
    x = (0x2B5 * n) % (1 << n)
    spec = wl.qft(n, x)
    got, _ = engine_state(sq, spec, "f64")
    assert np.abs(got - cf.qft_basis(n, x)).max() < TOL_F64
    got32, _ = engine_state(sq, spec, "f32")
    assert fidelity_gap(got32, got) < 1e-6


@pytest.mark.parametrize("n,warp_bits", [(18, 0), (18, 3), (22, 2)])
def test_qft_phase_terms_across_passes(sq, n, warp_bits):
    """Larger QFTs: their controlled phases pair tile bits with thread and
    non-tile bits over several passes, as compact phase terms (FP64 and FP32)."""
    x = (0x1F3D5 * n) % (1 << n)
    spec = wl.qft(n, x)
    want = cf.qft_basis(n, x)
    got, _ = engine_state(sq, spec, "f64", warp_bits=warp_bits)
    assert np.abs(got - want).max() < TOL_F64
    got32, _ = engine_state(sq, spec, "f32", warp_bits=warp_bits)
    assert fidelity_gap(got32, want) < 1e-6


def test_iterations_replay(sq):
    """Applying the PT list `iterations` times equals unrolling it."""
    n = 13
    spec = random_gate_circuit_spec(n, 40, seed=5)
    init = random_state(n, seed=9)
    got, _ = engine_state(sq, spec, "f64", init=init, iterations=3)
    c = spec.build(cl.Circuit())
    want = cpu.run_serial(init, n, c.as_arrays(), iterations=3)
    assert np.abs(got - want).max() < TOL_F64


def test_fp32_renormalisation(sq):
    """FP32 plans rescale to unit norm between passes; the result stays within tolerance."""
    n = 16
    spec = wl.random_layered(n, 8, seed=2)
    got64, _ = engine_state(sq, spec, "f64")
    got32, stats = engine_state(sq, spec, "f32", renorm_every=1)
    assert stats["passes"] > 2
    assert fidelity_gap(got32, got64) < 1e-6
    assert abs(np.vdot(got32, got32).real - 1.0) < 1e-5
