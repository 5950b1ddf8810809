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


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_autotune_keeps_results(sq, prec):
    """The autotuner tries every tile size and resident-low-bit count and
    leaves the batch finalized with the fastest; results still match the
    oracle afterwards."""
    specs = mixed_specs(41, 12, 8, 14)
    b = sq.Batch(prec, 2)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, spec.init_index)
    b.finalize().run()  # a finalized, already-run batch may be retuned
    pick = b.autotune()
    assert 0 <= pick["warp_bits"] <= 3 and pick["low_bits"] in (3, 4, 5) and pick["ms"] > 0
    b.run()
    sq.synchronize()
    b.check()
    for j, spec in enumerate(specs):
        got = b.state(j).download()
        assert np.abs(got - oracle_state(spec, prec)).max() < (TOL_F64 if prec == "f64" else TOL_F32), spec.name


def test_batch_set_inputs(sq):
    """New initial basis states per run (hgm_batch_set_inputs) give the
    results of those inputs; an index outside a job's state is refused."""
    rng = np.random.default_rng(9)
    ns = [int(x) for x in rng.integers(9, 14, 10)]
    specs = [wl.qft(n, 0) for n in ns]
    b = sq.Batch("f64", 1)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, 0)
    b.finalize()
    for rep in range(2):
        inputs = np.array([int(rng.integers(1 << n)) for n in ns], dtype=np.int64)
        b.set_inputs(inputs).run()
        sq.synchronize()
        for j, (spec, x) in enumerate(zip(specs, inputs)):
            spec_x = wl.qft(spec.qubits, int(x))
            assert np.abs(b.state(j).download() - oracle_state(spec_x, "f64")).max() < TOL_F64, (rep, j)
    bad = np.zeros(len(ns), dtype=np.int64)
    bad[3] = 1 << ns[3]
    with pytest.raises(sq.HgmError):
        b.set_inputs(bad)


def test_batch_bounded_wait_times_out(sq):
    """The persistent kernel's dependency wait is bounded: a task made to wait
    for a completion that never comes (injected on the host, with a 1 ms
    limit) gives up, the run ends and hgm_batch_check reports
    HGM_ERR_TIMEOUT; with the normal table restored the next run is clean and
    its results match the oracle again."""
    specs = [wl.random_layered(16, 6, seed=61), wl.random_layered(15, 6, seed=62)]
    b = sq.Batch("f64", 1)
    for spec in specs:
        b.add(spec.build(sq.Circuit()), spec.qubits, spec.init_index)
    b.finalize()
    ntasks = b.size()["tasks"]
    stalled = None
    for t in range(len(specs), ntasks):  # wave 0 has no dependencies
        try:
            b.inject_stall(t, 1_000_000)
            stalled = t
            break
        except sq.HgmError:
            continue
    assert stalled is not None
    b.run()
    sq.synchronize()
    with pytest.raises(sq.HgmError) as e:
        b.check()
    assert e.value.code == 5  # HGM_ERR_TIMEOUT
    b.inject_stall(-1)
    b.run()
    sq.synchronize()
    b.check()
    for j, spec in enumerate(specs):
        assert np.abs(b.state(j).download() - oracle_state(spec, "f64")).max() < TOL_F64
