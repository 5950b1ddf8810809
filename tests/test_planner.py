"""Planner checks on the CPU: the encoded passes, emulated with numpy
(tests/plan_emulator.py), reproduce the oracle; plans respect their limits.
"""
import numpy as np
import pytest

import simulador_quantico_b200 as sq
from simulador_quantico_b200 import workloads as wl
from tests import plan_emulator as emu
from tests.helpers import oracle_state, random_gate_circuit_spec, random_state


@pytest.mark.parametrize("n", [5, 9, 10, 11, 12, 14])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
@pytest.mark.parametrize("fuse", [0, 1, 2])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_emulated_plan_matches_oracle(n, warp_bits, fuse, prec):
    R = emu.REG_BITS[prec]
    if n >= 5 + R and 5 + R + warp_bits > n:
        pytest.skip("tile larger than state")
    if n < 5 + R and warp_bits:
        pytest.skip("small-state path")
    spec = random_gate_circuit_spec(n, 5 * n, seed=1000 + n * 10 + warp_bits + 100 * fuse)
    init = random_state(n, seed=n)
    plan = sq.Plan(spec.build(sq.Circuit()), n, prec, warp_bits=warp_bits, fuse=fuse, renorm_every=0)
    got = emu.run(plan, prec, init)
    want = oracle_state(spec, "f64", init=init)
    assert np.abs(got - want).max() < (1e-12 if prec == "f64" else 1e-5)


@pytest.mark.parametrize("low_bits", [0, 2, 5])
def test_emulated_low_bits(low_bits):
    n = 13
    spec = random_gate_circuit_spec(n, 60, seed=low_bits)
    init = random_state(n, seed=1)
    plan = sq.Plan(spec.build(sq.Circuit()), n, "f64", low_bits=low_bits, warp_bits=2)
    assert np.abs(emu.run(plan, "f64", init) - oracle_state(spec, "f64", init=init)).max() < 1e-12


@pytest.mark.parametrize("builder", [lambda: wl.random_layered(13, 3, 5), lambda: wl.qft(12, 1234),
                                     lambda: wl.grover_reference(12, 99, 2), lambda: wl.hadamard_benchmark(14)])
def test_emulated_workloads(builder):
    spec = builder()
    n = spec.qubits
    plan = sq.Plan(spec.build(sq.Circuit()), n, "f64")
    init = np.zeros(1 << n, dtype=np.complex128)
    init[spec.init_index] = 1
    assert np.abs(emu.run(plan, "f64", init) - oracle_state(spec, "f64")).max() < 1e-12


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("low_bits,warp_bits", [(3, 0), (4, 3), (5, 1), (4, 2)])
def test_emulated_tile_settings(prec, low_bits, warp_bits):
    """The batched autotuner's settings (always-resident low bits 3..5, warp
    bits 0..3): every layout keeps its conflict-free and coalescing rules
    (checked inside the emulator) and the plan reproduces the oracle, for a
    random-gate circuit and for a QFT (compact phase terms)."""
    n = 15
    tol = 1e-12 if prec == "f64" else 2e-5
    for spec in (random_gate_circuit_spec(n, 70, seed=low_bits * 10 + warp_bits), wl.qft(n, 4321)):
        plan = sq.Plan(spec.build(sq.Circuit()), n, prec, low_bits=low_bits, warp_bits=warp_bits, renorm_every=0)
        if spec.name == "qft":
            init = np.zeros(1 << n, dtype=np.complex128)
            init[spec.init_index] = 1
        else:
            init = random_state(n, seed=3)
        got = emu.run(plan, prec, init)
        assert np.abs(got - oracle_state(spec, "f64", init=init)).max() < tol, spec.name


def test_emulated_fp32_encoding():
    n = 12
    spec = random_gate_circuit_spec(n, 50, seed=9)
    init = random_state(n, seed=2)
    plan = sq.Plan(spec.build(sq.Circuit()), n, "f32", renorm_every=0)
    got = emu.run(plan, "f32", init)
    assert np.abs(got - oracle_state(spec, "f64", init=init)).max() < 1e-5


def test_plan_pass_counts():
    """Passes per 30-qubit random layer stay small (planner quality)."""
    spec = wl.random_layered(30, 4, seed=1)
    p = sq.Plan(spec.build(sq.Circuit()), 30, "f64")
    s = p.stats()
    assert s["ops"] == 4 * 45  # Rz.Ry fused per qubit + 15 CNOTs per layer
    assert s["passes"] <= 4 * 3
    p2 = sq.Plan(spec.build(sq.Circuit()), 30, "f64", fuse=2)
    assert p2.stats()["ops"] == 4 * 75  # fuse=2: Rz and Ry kept apart
    assert p2.stats()["passes"] <= 4 * 3


def test_fusion_merges_adjacent():
    """Adjacent gates on one target merge (H.H and Rz.Rz.Ry become one record
    each; with fuse=2 a pure phase next to a real gate stays apart); a gate on
    another qubit in between does not block it."""
    h = np.array([[1, 1], [1, -1]]) / np.sqrt(2)

    def rz(t):
        return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])

    def ry(t):
        return np.array([[np.cos(t / 2), -np.sin(t / 2)], [np.sin(t / 2), np.cos(t / 2)]])

    c = sq.Circuit()
    c.append_op(0, 0, 0, h)
    c.append_op(3, 0, 0, h)
    c.append_op(0, 0, 0, h)
    assert sq.Plan(c, 12, "f64").stats()["ops"] == 2
    c = sq.Circuit()
    for m in (rz(0.3), rz(0.5), ry(0.7)):
        c.append_op(0, 0, 0, m)
    # all three merge; with fuse=2 the pure phase (Rz.Rz) and the real Ry stay apart
    assert sq.Plan(c, 12, "f64").stats()["ops"] == 1
    assert sq.Plan(c, 12, "f64", fuse=2).stats()["ops"] == 2


def test_grover_plan_fast():
    """The unrolled 27-qubit Grover (grover.out 27, ~682k PTs) plans in seconds."""
    import time

    spec = wl.grover_reference(27, 42)
    c = spec.build(sq.Circuit())
    assert len(c) == 27 + 106 * 6433
    t0 = time.time()
    p = sq.Plan(c, 27, "f64")
    dt = time.time() - t0
    assert dt < 20.0
    assert p.stats()["passes"] < 6 * 6433


def test_randomized_plans():
    """Seeded random mix of precisions, tile settings, fusion and circuit
    families: every emulated plan (layout rules checked inside) reproduces
    the oracle."""
    rng = np.random.default_rng(20261203)
    for case in range(40):
        prec = ["f64", "f32"][case % 2]
        R = 4 if prec == "f64" else 5
        n = int(rng.integers(5 + R, 14))
        W = min(int(rng.integers(0, 4)), n - 5 - R)
        lb = int(rng.integers(0, 6))
        kind = case % 4
        if kind == 0:
            spec = random_gate_circuit_spec(n, int(rng.integers(5, 6 * n)), seed=int(rng.integers(1 << 30)),
                                            max_controls=int(rng.integers(0, 4)))
            init = random_state(n, seed=case)
        else:
            spec = [None, lambda: wl.qft(n, int(rng.integers(1 << n))),
                    lambda: wl.random_layered(n, int(rng.integers(1, 4)), case),
                    lambda: wl.grover_search(n, int(rng.integers(1 << n)), iterations=2)][kind]()
            init = np.zeros(1 << n, dtype=np.complex128)
            init[spec.init_index] = 1
        plan = sq.Plan(spec.build(sq.Circuit()), n, prec, warp_bits=W, low_bits=lb, fuse=case % 3,
                       renorm_every=0)
        got = emu.run(plan, prec, init)
        want = oracle_state(spec, "f64", init=init)
        assert np.abs(got - want).max() < (1e-11 if prec == "f64" else 5e-5), (case, prec, n, W, lb, spec.name)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("split", [0, 1])
def test_emulated_split_layers(prec, split):
    """Layers of complex gates as phase, real gate, phase (K_LAYER_SPLIT) with
    the gates' scalar factors applied once at the end: the records reproduce
    the oracle, and split plans hold split layers exactly when asked to."""
    n = 14
    tol = 1e-12 if prec == "f64" else 2e-5
    spec = wl.random_layered(n, 4, seed=31)
    plan = sq.Plan(spec.build(sq.Circuit()), n, prec, split_layers=split, renorm_every=0)
    kinds = {int(o["kind"]) for o in emu.export(plan, prec)["ops"]}
    assert (emu.K_LAYER_SPLIT in kinds) == bool(split)
    init = random_state(n, seed=4)
    assert np.abs(emu.run(plan, prec, init) - oracle_state(spec, "f64", init=init)).max() < tol


def test_split_layer_gate_forms():
    """Gates with the split form (Rz Ry, Ry Rz, Rz Ry Rz, a general unitary,
    a real matrix times a phase) go out as split layers; a complex matrix
    without it (a column whose entries differ in phase by other than 0 or pi)
    keeps the dense form; results match the oracle either way."""
    n = 12
    rng = np.random.default_rng(5)

    def rz(t):
        return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])

    def ry(t):
        return np.array([[np.cos(t / 2), -np.sin(t / 2)], [np.sin(t / 2), np.cos(t / 2)]])

    def unitary():
        q, r = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
        return q * (np.diag(r) / np.abs(np.diag(r)))

    forms = [ry(0.4) @ rz(1.1), rz(0.9) @ ry(2.2), rz(0.3) @ ry(1.3) @ rz(2.9), unitary(),
             np.exp(0.7j) * ry(0.8)]
    for m in forms:
        c = sq.Circuit()
        for q in range(n):
            c.append_op(q, 0, 0, m)
        plan = sq.Plan(c, n, "f64", split_layers=1)
        kinds = [int(o["kind"]) for o in emu.export(plan, "f64")["ops"]]
        assert emu.K_LAYER_SPLIT in kinds and emu.K_LAYER not in kinds
        init = random_state(n, seed=6)
        want = init.reshape([2] * n)
        for q in range(n):  # index bit q is axis n-1-q
            want = np.moveaxis(np.tensordot(m, want, axes=([1], [n - 1 - q])), 0, n - 1 - q)
        assert np.abs(emu.run(plan, "f64", init) - want.reshape(-1)).max() < 1e-12
    bad = np.array([[1.0, 1.0], [1j, 2.0]]) / 2.0
    c = sq.Circuit()
    for q in range(n):
        c.append_op(q, 0, 0, bad)
    kinds = [int(o["kind"]) for o in emu.export(sq.Plan(c, n, "f64", split_layers=1), "f64")["ops"]]
    assert emu.K_LAYER in kinds and emu.K_LAYER_SPLIT not in kinds


@pytest.mark.parametrize("n", [9, 10, 12, 14])
@pytest.mark.parametrize("warp_bits", [0, 1, 2, 3])
def test_emulated_f32_sixteen_registers(n, warp_bits):
    """FP32 plans with 16 amplitudes a thread (reg_bits = 4)."""
    if 9 + warp_bits > n:
        pytest.skip("tile larger than state")
    spec = random_gate_circuit_spec(n, 5 * n, seed=77 + n + warp_bits)
    init = random_state(n, seed=n)
    plan = sq.Plan(spec.build(sq.Circuit()), n, "f32", reg_bits=4, warp_bits=warp_bits, renorm_every=0)
    assert plan.stats()["reg_bits"] == 4
    assert np.abs(emu.run(plan, "f32", init) - oracle_state(spec, "f64", init=init)).max() < 2e-5


def test_reg_bits_validated():
    spec = random_gate_circuit_spec(12, 10, seed=1)
    for prec, bad in (("f64", 5), ("f64", 3), ("f32", 3), ("f32", 6)):
        with pytest.raises(Exception):
            sq.Plan(spec.build(sq.Circuit()), 12, prec, reg_bits=bad)
    assert sq.Plan(spec.build(sq.Circuit()), 12, "f32").stats()["reg_bits"] == 5
    assert sq.Plan(spec.build(sq.Circuit()), 12, "f64").stats()["reg_bits"] == 4
