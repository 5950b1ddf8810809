"""Serving mode on the GPU: continuous batching with byte-based admission.

Every served result must equal the same circuit run alone (within the FP32
tolerance), whatever else ran with it; admission never exceeds the budget;
a state larger than the budget is refused.
"""
import math
import time

import numpy as np
import pytest

from oracle import closed_forms as cf
from simulador_quantico_b200 import workloads as wl
from tests.helpers import engine_state, fidelity_gap, oracle_state

pytestmark = pytest.mark.gpu


def request_mix(seed, count):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        u = rng.random()
        if u < 0.6:
            spec = wl.random_layered(int(rng.integers(10, 17)), 4, seed=seed * 1000 + i)
            mask = 0
        elif u < 0.9:
            n = int(rng.integers(10, 17))
            spec = wl.qft(n, int(rng.integers(1 << n)))
            mask = (1 << n) - 1
        else:
            m = int(rng.integers(8, 13))
            spec = wl.grover_search(m, int(rng.integers(1 << m)))
            mask = (1 << m) - 1
        reqs.append((spec, mask))
    return reqs


@pytest.mark.parametrize("order", ["arrival", "work_first"])
def test_served_results_equal_alone(sq, order):
    reqs = request_mix(11, 40)
    srv = sq.Server("f32", budget_bytes=1 << 30, max_inflight=8, keep_states=True, order=order)
    ids = {}
    for spec, mask in reqs:
        rid = srv.submit(spec.build(sq.Circuit()), spec.qubits, spec.init_index, mask)
        ids[rid] = (spec, mask)
    results = srv.drain(len(reqs))
    assert all(r["status"] == 0 for r in results)
    for r in results:
        spec, mask = ids[r["id"]]
        got = srv.result_state(r["id"]).download()
        alone, _ = engine_state(sq, spec, "f32")
        assert np.abs(got - alone).max() < 1e-6, spec.name
        want64 = oracle_state(spec, "f64")
        assert fidelity_gap(got, want64) < 1e-6
        assert abs(r["norm"] - 1.0) < 1e-4  # FP32 norm drift over ~200 gates, FP64-accumulated
        if spec.name == "grover":
            assert r["argmax"] == spec.meta["search_value"]
        if spec.name == "qft":
            assert abs(r["pmax"] - 2.0 ** -spec.qubits) < 1e-6  # uniform magnitudes
        srv.release(r["id"])
    srv.close()


@pytest.mark.parametrize("order", ["arrival", "work_first"])
def test_admission_respects_budget(sq, order):
    budget = 4 * (8 << 16)  # four 16-qubit FP32 states
    srv = sq.Server("f32", budget_bytes=budget, max_inflight=16, order=order)
    n = 16
    for i in range(12):
        spec = wl.random_layered(n, 6, seed=i)
        srv.submit(spec.build(sq.Circuit()), n)
    seen = 0
    t0 = time.time()
    while seen < 12 and time.time() - t0 < 60:
        p = srv.pending()
        assert p["bytes_in_use"] <= budget
        assert p["inflight"] <= 4
        seen += len(srv.poll(wait_ms=1))
    assert seen == 12
    srv.close()


def test_oversized_request_refused(sq):
    srv = sq.Server("f64", budget_bytes=1 << 20)
    spec = wl.hadamard_benchmark(17)  # 2 MiB FP64 state
    with pytest.raises(sq.HgmError) as e:
        srv.submit(spec.build(sq.Circuit()), 17)
    assert e.value.code == 6
    srv.close()


def test_fp64_server_matches_oracle(sq):
    reqs = request_mix(5, 12)
    srv = sq.Server("f64", budget_bytes=1 << 30, max_inflight=4, keep_states=True)
    ids = {srv.submit(spec.build(sq.Circuit()), spec.qubits, spec.init_index, mask): spec for spec, mask in reqs}
    for r in srv.drain(len(reqs)):
        spec = ids[r["id"]]
        got = srv.result_state(r["id"]).download()
        assert np.abs(got - oracle_state(spec, "f64")).max() < 1e-12
        srv.release(r["id"])
    srv.close()


def test_submit_plan_matches_submit(sq):
    """A request queued as a prebuilt plan (hgm_server_submit_plan) gives the
    same result as the same circuit submitted for the server to plan; a plan
    of the wrong precision is refused."""
    reqs = request_mix(23, 12)
    srv = sq.Server("f32", budget_bytes=1 << 30, max_inflight=4, keep_states=True)
    plans, ids = [], {}
    for spec, mask in reqs:
        c = spec.build(sq.Circuit())
        p = sq.Plan(c, spec.qubits, "f32")
        plans.append(p)
        ids[srv.submit_plan(p, spec.init_index, mask)] = ("plan", spec)
        ids[srv.submit(c, spec.qubits, spec.init_index, mask)] = ("circuit", spec)
    results = {r["id"]: r for r in srv.drain(2 * len(reqs))}
    assert all(r["status"] == 0 for r in results.values())
    rids = sorted(ids)
    for a, b in zip(rids[0::2], rids[1::2]):
        assert ids[a][0] == "plan" and ids[b][0] == "circuit"
        ga, gb = srv.result_state(a).download(), srv.result_state(b).download()
        assert np.array_equal(ga, gb), ids[a][1].name
        assert results[a]["argmax"] == results[b]["argmax"]
    with pytest.raises(sq.HgmError):
        srv.submit_plan(sq.Plan(reqs[0][0].build(sq.Circuit()), reqs[0][0].qubits, "f64"))
    srv.close()


def test_state_buffers_recycled_within_budget(sq):
    """Finished states' buffers are reused by later requests of the same
    size, and cached buffers of other sizes are evicted when a new size would
    not fit the budget; every result is still exact (each request
    re-initialises the buffer it gets) and admission stays within budget."""
    budget = 3 * (8 << 16)  # three 16-qubit FP32 states
    srv = sq.Server("f32", budget_bytes=budget, max_inflight=4)
    sizes = [16, 15, 16, 14, 16, 15, 13, 16, 14, 15, 16, 12] * 2
    ids = {}
    for i, n in enumerate(sizes):
        spec = wl.grover_search(n, (37 * i + 5) % (1 << n), iterations=3) if i % 2 else wl.qft(n, (91 * i) % (1 << n))
        ids[srv.submit(spec.build(sq.Circuit()), n, spec.init_index, (1 << n) - 1)] = spec
        p = srv.pending()
        assert p["bytes_in_use"] <= budget
    results = srv.drain(len(sizes))
    assert all(r["status"] == 0 for r in results)
    for r in results:
        spec = ids[r["id"]]
        assert abs(r["norm"] - 1.0) < 1e-4
        if spec.name == "qft":
            assert abs(r["pmax"] - 2.0 ** -spec.qubits) < 1e-6
        else:
            want = oracle_state(spec, "f64")
            assert r["argmax"] == int(np.argmax(np.abs(want) ** 2))
    srv.close()


def test_work_first_admits_largest(sq):
    """With one slot, the work-first order admits the queued request with the
    most work (state bytes x passes) next, not the oldest."""
    srv = sq.Server("f32", budget_bytes=1 << 30, max_inflight=1, order="work_first")
    first = wl.random_layered(20, 30, seed=1)  # holds the slot while the rest queue
    srv.submit_plan(sq.Plan(first.build(sq.Circuit()), 20, "f32").upload(), 0)
    small = wl.random_layered(12, 2, seed=2)
    big = wl.random_layered(18, 8, seed=3)
    plans = [sq.Plan(small.build(sq.Circuit()), 12, "f32").upload(), sq.Plan(big.build(sq.Circuit()), 18, "f32").upload()]
    rid_small = srv.submit_plan(plans[0], 0)
    rid_big = srv.submit_plan(plans[1], 0)
    res = srv.drain(3)
    assert all(r["status"] == 0 for r in res)
    queued = {r["id"]: r["queue_s"] for r in res}  # submit -> admitted
    assert queued[rid_big] < queued[rid_small]
    srv.close()


def test_plan_freed_while_queued(sq):
    """A plan whose Python object is gone right after hgm_server_submit_plan
    (hgm_plan_free while the request is queued behind a long one) stays valid
    until the request is done: the request leases it."""
    import gc

    srv = sq.Server("f32", budget_bytes=1 << 30, max_inflight=1)
    hold = sq.Plan(wl.random_layered(20, 30, seed=5).build(sq.Circuit()), 20, "f32").upload()
    srv.submit_plan(hold, 0)
    spec = wl.qft(14, 1234)
    rid = srv.submit_plan(sq.Plan(spec.build(sq.Circuit()), 14, "f32").upload(), spec.init_index, (1 << 14) - 1)
    gc.collect()
    res = {r["id"]: r for r in srv.drain(2)}
    assert res[rid]["status"] == 0
    assert abs(res[rid]["pmax"] - 2.0 ** -14) < 1e-6
    srv.close()
