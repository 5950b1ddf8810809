"""The reference's GPU-backend C-ABI (GpuExecutionWrapper & co.) on the GPU.

Calls libhgm_dropin_{f32,f64}.so exactly as the reference's DGM::execute
does (src/core/dgm_core.cpp:255-257): host state in, PT** list, tuning
arguments, iterations; state updated in place.  When oracle/_ref holds the
reference's own objects linked against the drop-in, the reference's DGM
itself drives the engine and is compared with its own t_CPU backend.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import closed_forms as cf
from oracle import cpu
from simulador_quantico_b200 import workloads as wl
from tests.helpers import TOL_F32, TOL_F64, oracle_state, random_gate_circuit_spec, random_state

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def run_wrapper(sq, spec, prec, init, iterations=1, tuning=(4, 8, 1, 64, 2)):
    L = sq.load_dropin(prec)
    assert L.setDevice(0) is False  # CUDA error as bool: false on success
    c = spec.build(sq.Circuit())
    pts = c.ref_pts(prec)
    dt = np.complex128 if prec == "f64" else np.complex64
    host = np.ascontiguousarray(init.astype(dt))
    ret = L.GpuExecutionWrapper(host.ctypes.data, pts, spec.qubits, *tuning, iterations)
    assert ret == host.ctypes.data  # same pointer returned, updated in place
    return host


@pytest.mark.parametrize("n", [6, 12, 17])
def test_wrapper_f64(sq, n):
    spec = random_gate_circuit_spec(n, 8 * n, seed=31 + n)
    init = random_state(n, seed=n)
    got = run_wrapper(sq, spec, "f64", init, iterations=2)
    c = spec.build(__import__("oracle.circuit_lang", fromlist=["Circuit"]).Circuit())
    want = cpu.run_serial(init, n, c.as_arrays(), iterations=2)
    assert np.abs(got - want).max() < TOL_F64


@pytest.mark.parametrize("n", [6, 14])
def test_wrapper_f32(sq, n):
    spec = random_gate_circuit_spec(n, 6 * n, seed=77 + n)
    init = random_state(n, seed=n, dtype=np.complex64)
    got = run_wrapper(sq, spec, "f32", init)
    want = oracle_state(spec, "f32", init=init)
    assert np.abs(got - want).max() < TOL_F32


def test_wrapper_hadamard_20(sq):
    spec = wl.hadamard_benchmark(20, 3)
    got = run_wrapper(sq, spec, "f64", cpu.basis_state(20, 0))
    assert np.abs(got - cf.hadamard_all(20)).max() < TOL_F64


def test_hybrid_entry_points_refuse(sq):
    L = sq.load_dropin("f64")
    buf = np.zeros(16, dtype=np.complex128)
    assert L.ProjectState(buf.ctypes.data, 4, 4, 0, 15, 1) is False
    assert L.GetState(buf.ctypes.data, 4, 4, 0, 15, 1) is False


@pytest.mark.skipif(not cpu.ref_available("f64", dropin=True), reason="reference objects not built here")
@pytest.mark.parametrize("n", [11, 14])
def test_reference_dgm_drives_engine(sq, n):
    """The reference's own DGM (FP64-widened) with t_GPU linked to this engine vs its t_CPU."""
    w = 37 % (1 << (n - 1))
    spec = wl.grover_reference(n, w, iterations=4)
    results = {}
    for name, dropin, exec_type in (("gpu", True, cpu.RefDGM.T_GPU), ("cpu", False, cpu.RefDGM.T_CPU)):
        r = cpu.RefDGM(n, "f64", dropin=dropin)
        r.tuning(exec_type)
        r.set_memory_value(spec.init_index)
        for steps, it, reset in spec.calls:
            r.set_function(steps, it, reset)
        r.execute(1)
        results[name] = r.state()
        r.close()
    assert np.abs(results["gpu"] - results["cpu"]).max() < TOL_F64


@pytest.mark.skipif(not (REF / "general_b200_f64.out").exists(), reason="reference CLIs not built here")
@pytest.mark.parametrize("prec,n,amp", [("f64", 10, "0.031250"), ("f64", 18, "0.001953"), ("f32", 14, "0.007812")])
def test_general_out_unchanged(sq, prec, n, amp):
    """tests/smoke_test.sh:90-95: general.out <n> 2 1 prints amplitude 0 = 2^-n/2."""
    out = subprocess.run([str(REF / f"general_b200_{prec}.out"), str(n), "2", "1"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    first = out.stdout.splitlines()[0].split()
    assert first[1] == amp


@pytest.mark.skipif(not (REF / "grover_b200_f64.out").exists(), reason="reference CLIs not built here")
def test_grover_out_unchanged(sq):
    """tests/smoke_test.sh:117: grover.out 12 2 1 finds the search value."""
    hits = 0
    for _ in range(3):
        out = subprocess.run([str(REF / "grover_b200_f64.out"), "12", "2", "1", "64", "2", "8", "10"],
                             capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stdout + out.stderr
        hits += "Found value: 10" in out.stdout
    assert hits >= 2


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_shor_out_unchanged(sq, prec):
    """tests/smoke_test.sh:114-120: shor.out 15 2 1 (t_GPU) runs without a
    crash and finds the factors of 57 at least once in 16 runs (Shor's
    period finding is probabilistic; 2n executeFunction + measure rounds,
    each a GpuExecutionWrapper call on the host state)."""
    exe = REF / f"shor_b200_{prec}.out"
    if not exe.exists():
        pytest.skip("reference CLIs not linked (oracle/build_ref.sh)")
    found = 0
    for _ in range(16):
        out = subprocess.run([str(exe), "15", "2", "1"], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0 and "Time:" in out.stdout, out.stdout + out.stderr
        if "Found factors: 3 -- 19" in out.stdout or "Found factors: 19 -- 3" in out.stdout:
            found += 1
            break
    assert found >= 1


def test_wrapper_interleaved_sizes(sq):
    """The drop-in keeps one device state per qubit count between calls;
    calls that alternate between sizes still get exact results."""
    for i, n in enumerate([12, 14, 12, 16, 14, 12]):
        spec = random_gate_circuit_spec(n, 4 * n, seed=300 + i)
        init = random_state(n, seed=500 + i)
        got = run_wrapper(sq, spec, "f64", init)
        c = spec.build(__import__("oracle.circuit_lang", fromlist=["Circuit"]).Circuit())
        want = cpu.run_serial(init, n, c.as_arrays())
        assert np.abs(got - want).max() < TOL_F64, n


def test_wrapper_plan_cache(sq):
    """GpuExecutionWrapper keeps the plans of recent PT lists: the same list on
    new inputs, a list of the same length with one matrix changed, and more
    lists than the cache holds all give the oracle's results."""
    n = 13
    L = sq.load_dropin("f64")
    assert L.setDevice(0) is False
    specs = [random_gate_circuit_spec(n, 40, seed=900 + k) for k in range(10)]
    twin = random_gate_circuit_spec(n, 40, seed=900)
    first = next(iter(twin.gates))
    twin.gates[first] = [0, 1j, 1j, 0]  # same targets and controls, another matrix
    for rep in range(2):
        for k, spec in enumerate(specs[:3] + [twin] + specs[3:]):
            init = random_state(n, seed=rep * 100 + k)
            c = spec.build(sq.Circuit())
            host = init.copy()
            L.GpuExecutionWrapper(host.ctypes.data, c.ref_pts("f64"), n, 4, 8, 1, 64, 2, 1)
            want = oracle_state(spec, "f64", init=init)
            assert np.abs(host - want).max() < TOL_F64, (rep, k)
