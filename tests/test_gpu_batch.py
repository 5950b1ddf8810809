"""Batched mode on the GPU: many circuits of uneven size in one persistent kernel.

Each batched result must equal the same circuit run alone through the plain
pass path (and the oracle), within the stated tolerance: FP64 1e-12, FP32
2e-5 against the FP32 oracle.
"""
import numpy as np
import pytest

from simulador_quantico_b200 import workloads as wl
from tests.helpers import TOL_F32, TOL_F64, engine_state, oracle_state

pytestmark = pytest.mark.gpu


def mixed_specs(seed, count, lo, hi):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.integers(lo, hi + 1))
        if i % 2:
            specs.append(wl.qft(n, int(rng.integers(1 << n))))
        else:
            specs.append(wl.random_layered(n, 3, seed=seed * 100 + i))
    return specs


@pytest.mark.parametrize("prec,warp_bits", [("f64", 0), ("f64", 2), ("f32", 1), ("f32", 3)])
def test_batch_matches_oracle(sq, prec, warp_bits):
    specs = mixed_specs(7 + warp_bits, 24, 6, 15)
    b = sq.Batch(prec, warp_bits)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, spec.init_index)
    b.finalize()
    for rep in range(2):  # the graph replays from the initial states every run
        b.run()
        sq.synchronize()
        b.check()
        for j, spec in enumerate(specs):
            got = b.state(j).download()
            want = oracle_state(spec, prec)
            assert np.abs(got - want).max() < (TOL_F64 if prec == "f64" else TOL_F32), (rep, j, spec.name, spec.qubits)


def test_batch_equals_alone(sq):
    """A circuit's batched result is the one it gets alone (same plan, same tile order per amplitude)."""
    specs = mixed_specs(3, 16, 10, 17)
    b = sq.Batch("f32", 2)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, spec.init_index)
    b.finalize().run()
    sq.synchronize()
    for j, spec in enumerate(specs):
        alone, _ = engine_state(sq, spec, "f32", warp_bits=2, renorm_every=0)
        got = b.state(j).download()
        assert np.abs(got - alone).max() < 1e-6


def test_batch_size_report(sq):
    specs = mixed_specs(5, 8, 12, 16)
    b = sq.Batch("f64", 1)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, spec.init_index)
    b.finalize()
    s = b.size()
    assert s["jobs"] == 8 and s["tasks"] >= 8 and s["items"] >= s["tasks"]
    assert s["arena_bytes"] == sum(16 << spec.qubits for spec in specs)
