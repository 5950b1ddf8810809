"""Benchmark for the B200 state-vector engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

Workloads (synthetic, seeded):
  served   the serving stream: a seeded request mix (60% random layered
           circuits of 12-26 qubits, 30% QFTs of 16-28, 10% Grover searches
           of 14-20) served by the continuous-batching server in FP32 with
           FP64 norm checks; metric served circuits/s; default 20 timed steps
           of 48 requests after 5 warm-up steps
  batched  512 circuits of 10-22 qubits (half QFTs, half random layered) in
           one persistent kernel replayed from a CUDA graph, FP32 (value) and
           FP64, autotuned; metric batched circuits/s
  hadamard one gate layer, H on every qubit of a 30-qubit FP64 state (the
           Hadamard benchmark's shape); metric gate-layers/s
  layered  a 30-qubit, 40-layer random Rz/Ry + CNOT circuit in FP64; metric
           gate-layers/s (one step = the whole circuit)
  qft      the textbook QFT of a basis state, 28 qubits FP32 by default;
           metric QFT circuits/s
  grover   Grover search, 26 qubits FP64, marked index 42 (the phase
           oracle + diffusion form, no ancilla); metric Grover iterations/s
           (one step = 64 iterations); the full 6433-iteration search is run
           after the timed steps and its argmax checked

Timing: W untimed warm-up steps, then K steps between a barrier and a device
synchronize on both sides, timed with CUDA events on the library stream;
the max over ranks is reported.  With N > 1 every rank runs an independent
replica of the workload on its own GPU (no collective on the data path):
value = units of all ranks / max time.  The state passes are larger than L2
(126 MB) for layered and grover, so no cache flush is needed between steps.

--impl reference times the reference's own CPU engine (t_PAR_CPU,
PCpuExecution1, built by oracle/build_ref.sh into oracle/_ref) on a bounded
sample of the same workload with every host thread, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

# one hardware queue per server slot (16 streams); set before any CUDA context
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0

# DRAM bytes read + written per pass-kernel launch, over the algorithmic 2*S,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of two
# passes of the 26-qubit random layered circuit (FP32 1.017 GB and FP64
# 2.093 GB per launch against 1.074 / 2.147 GB) and of two passes of the
# 28-qubit Hadamard layer (8.555 GB against 8.590 GB).  Writes come out a
# little short because the last lines are still in L2 when the launch ends.
TRAFFIC_OVER_ALGO = {"f32": 0.947, "f64": 0.975, "f64_hadamard": 0.996}


_WL = None


def _workloads():
    """The circuit builders (simulador_quantico_b200/workloads.py), loaded by path: they need only numpy, and
    the reference arm must not import the engine package, whose import loads the CUDA library."""
    global _WL
    if _WL is None:
        import importlib.util

        name = "hgm_bench_workloads"
        spec = importlib.util.spec_from_file_location(name, ROOT / "simulador_quantico_b200" / "workloads.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
        _WL = mod
    return _WL


def hbm_peak():
    try:
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only: a barrier and a max of timings)
# ---------------------------------------------------------------------------

class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, name in enumerate(names):
                if s[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def run_timed(dist, sq, step, steps, warmup):
    """W warm-up steps, then K timed steps with CUDA events (device time)."""
    for _ in range(warmup):
        step()
    sq.synchronize()
    dist.barrier()
    sq.synchronize()
    launches0 = sq.kernel_launches()
    with sq.Timer() as t:
        for _ in range(steps):
            step()
    sq.synchronize()
    dist.barrier()
    return t.ms, sq.kernel_launches() - launches0


def workload_layered(args, dist, sq):
    wl = _workloads()

    n, layers, prec = args.qubits or 30, args.layers or 40, args.precision
    spec = wl.random_layered(n, layers, seed=2024)
    c = spec.build(sq.Circuit())
    plan = sq.Plan(c, n, prec)
    stats = plan.stats()
    st = sq.State(n, prec).set_basis(0)

    def step():
        st.execute(plan)

    with ClockSampler(dist.local_rank) as clk:
        ms, launches = run_timed(dist, sq, step, args.steps, args.warmup)
    ms_step = dist.max(ms / args.steps)
    S = st.nbytes
    value = dist.world * layers / (ms_step * 1e-3)
    # all pass launches in the timed region are pass kernels of this plan
    pass_ms = ms_step / stats["passes"]
    achieved = 2 * S / (pass_ms * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    # outside the timed region: the unitary circuit keeps the norm (FP64 reduction on the device)
    norm = st.norm()
    # end to end through the reference's C-ABI with host buffers (1 step)
    e2e = e2e_layered(dist, sq, spec, n, prec) if not args.skip_e2e else None
    st.free()
    line = base_line(args, dist, METRICS["layered"], value, "layers/s", ms_step, prec, config_for(args))
    line["plan"] = {"passes_per_step": stats["passes"], "ops_after_fusion": stats["ops"]}
    line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4),
                        "traffic": round(TRAFFIC_OVER_ALGO[prec] * 2 * S / 1e9, 3), "traffic_unit": "GB per launch",
                        "traffic_source": "ncu capture at 26 qubits, scaled to this state size",
                        "peak_source": peak_kind,
                        "kernel": "pass_kernel<%s,%d,%d>" % ({"f64": "double", "f32": "float"}[prec], stats["reg_bits"],
                                                             stats["warp_bits"]),
                        "algorithmic_bytes_per_launch": 2 * S}
    line["gpu_launches"] = launches
    line["clocks"] = clk.summary()
    line["norm_after"] = {"value": norm, "ok": bool(abs(norm - 1.0) < (1e-9 if prec == "f64" else 1e-3))}
    line["e2e"] = e2e
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_layered(args)
    return line


def e2e_layered(dist, sq, spec, n, prec):
    L = sq.load_dropin(prec)
    L.setDevice(dist.local_rank)
    c = spec.build(sq.Circuit())
    pts = c.ref_pts(prec)
    host = np.zeros(1 << n, dtype=np.complex64 if prec == "f32" else np.complex128)
    host[0] = 1.0
    # one untimed call first (device state, staging buffers, host pages), as a
    # DGM user's repeated execute calls would have
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, 1)
    host[:] = 0
    host[0] = 1.0
    t0 = time.perf_counter()
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, 1)
    dt = time.perf_counter() - t0
    dt = dist.max(dt)
    layers = spec.meta["layers"]
    return {"value": round(dist.world * layers / dt, 4), "unit": "layers/s", "h2d_bytes_per_step": int(host.nbytes),
            "d2h_bytes_per_step": int(host.nbytes), "path": "GpuExecutionWrapper (reference C-ABI), host state",
            "seconds": round(dt, 3)}


def cpu_baseline_layered(args, kind="reference"):
    """t_PAR_CPU on a bounded sample: 2 layers at 26 qubits, scaled by 2^(30-26)."""
    from oracle import cpu
    wl = _workloads()

    n_s, layers_s = 26, 2
    spec = wl.random_layered(n_s, layers_s, seed=2024)
    threads = os.cpu_count() or 1
    if cpu.ref_available("f64"):
        r = cpu.RefDGM(n_s, "f64")
        for name, m in spec.gates.items():
            r.add_gate(name, m)
        r.set_memory_value(0)
        for steps, it, reset in spec.calls:
            r.set_function(steps, it, reset)
        r.tuning(cpu.RefDGM.T_PAR_CPU, thread_count=threads)
        t0 = time.perf_counter()
        r.execute(1)
        dt = time.perf_counter() - t0
        r.close()
        kind = "reference"
    else:
        from oracle import circuit_lang as cl

        ops = spec.build(cl.Circuit()).as_arrays()
        s0 = cpu.basis_state(n_s, 0)
        t0 = time.perf_counter()
        cpu.run_regions(s0, n_s, ops, threads=threads)
        dt = time.perf_counter() - t0
        kind = "port"
    per_layer_30 = dt / layers_s * (1 << (30 - n_s))
    return {"value": round(1.0 / per_layer_30, 6), "unit": "layers/s", "cores": threads, "kind": kind,
            "sample": f"{layers_s} layers at {n_s} qubits FP64 t_PAR_CPU ({dt:.2f} s), scaled x{1 << (30 - n_s)} "
                      f"to 30 qubits"}



def workload_qft(args, dist, sq):
    """The textbook QFT of a basis state (the served mix's and the batch's QFT requests), 28 qubits FP32 by
    default (--qubits, --precision); one step = the circuit."""
    wl = _workloads()
    n, prec = args.qubits or 28, args.precision
    spec = wl.qft(n, 0x5A5A5A5 & ((1 << n) - 1))
    plan = sq.Plan(spec.build(sq.Circuit()), n, prec)
    stats = plan.stats()
    st = sq.State(n, prec).set_basis(spec.init_index)

    def step():
        st.execute(plan)

    with ClockSampler(dist.local_rank) as clk:
        ms, launches = run_timed(dist, sq, step, args.steps, args.warmup)
    ms_step = dist.max(ms / args.steps)
    S = st.nbytes
    st.free()
    peak, peak_kind = hbm_peak()
    achieved = stats["passes"] * 2 * S / (ms_step * 1e-3) / 1e9
    line = base_line(args, dist, METRICS["qft"], dist.world / (ms_step * 1e-3), "circuits/s", ms_step, prec,
                     config_for(args))
    line["plan"] = {"passes_per_step": stats["passes"], "ops_after_fusion": stats["ops"]}
    line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                        "kernel": "pass_kernel<%s,%d,%d>" % ({"f64": "double", "f32": "float"}[prec], stats["reg_bits"],
                                                             stats["warp_bits"]),
                        "algorithmic_bytes_per_launch": 2 * S}
    line["gpu_launches"] = launches
    line["clocks"] = clk.summary()
    return line


# ---------------------------------------------------------------------------
# one gate layer (config 1's shape, H on every qubit) at 30 qubits FP64
# ---------------------------------------------------------------------------

def workload_hadamard(args, dist, sq):
    """H on every qubit of a 30-qubit FP64 state: a gate layer with few gates per pass, so the pass kernel
    is bound by HBM rather than by its FP64 pipe.  One step = the layer."""
    wl = _workloads()

    n = args.qubits or 30
    spec = wl.hadamard_benchmark(n, iterations=1)
    c = spec.build(sq.Circuit())
    plan = sq.Plan(c, n, "f64")
    stats = plan.stats()
    st = sq.State(n, "f64").set_basis(0)

    def step():
        st.execute(plan)

    with ClockSampler(dist.local_rank) as clk:
        ms, launches = run_timed(dist, sq, step, args.steps, args.warmup)
    ms_step = dist.max(ms / args.steps)
    S = st.nbytes
    value = dist.world / (ms_step * 1e-3)
    achieved = stats["passes"] * 2 * S / (ms_step * 1e-3) / 1e9
    # outside the timed region: after an odd number of layers every amplitude is 2^(-n/2)
    runs = args.warmup + args.steps
    p0 = st.prob_one(0)
    st.free()
    peak, peak_kind = hbm_peak()
    line = base_line(args, dist, METRICS["hadamard"], value, "layers/s", ms_step, "f64", config_for(args))
    line["plan"] = {"passes_per_step": stats["passes"]}
    line["check"] = {"layers_applied": runs, "prob_one_bit0": p0,
                     "ok": bool(abs(p0 - (0.5 if runs % 2 else 0.0)) < 1e-9)}
    line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4),
                        "traffic": round(TRAFFIC_OVER_ALGO["f64_hadamard"] * 2 * S / 1e9, 3),
                        "traffic_unit": "GB per launch",
                        "traffic_source": "ncu capture of the 28-qubit Hadamard layer, scaled to this state size",
                        "peak_source": peak_kind,
                        "kernel": "pass_kernel<double,%d,%d>" % (stats["reg_bits"], stats["warp_bits"]),
                        "algorithmic_bytes_per_launch": 2 * S}
    line["gpu_launches"] = launches
    line["clocks"] = clk.summary()
    line["e2e"] = e2e_hadamard(dist, sq, c, n) if not args.skip_e2e else None
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_hadamard(args, n)
    return line


def e2e_hadamard(dist, sq, c, n):
    """The layer through the reference's C-ABI: GpuExecutionWrapper on a host state (16 GiB each way)."""
    L = sq.load_dropin("f64")
    L.setDevice(dist.local_rank)
    pts = c.ref_pts("f64")
    host = np.zeros(1 << n, dtype=np.complex128)
    host[0] = 1.0
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, 1)  # untimed first call
    host[:] = 0
    host[0] = 1.0
    t0 = time.perf_counter()
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, 1)
    dt = dist.max(time.perf_counter() - t0)
    ok = abs(host[0].real - 2.0 ** (-n / 2)) < 1e-12 and abs(host[-1].real - 2.0 ** (-n / 2)) < 1e-12
    return {"value": round(dist.world / dt, 4), "unit": "layers/s", "h2d_bytes_per_step": int(host.nbytes),
            "d2h_bytes_per_step": int(host.nbytes), "path": "GpuExecutionWrapper (reference C-ABI), host state",
            "seconds": round(dt, 3), "amplitudes_ok": bool(ok)}


def cpu_baseline_hadamard(args, n, n_s=26):
    """t_PAR_CPU: the layer at 26 qubits, scaled by 2^(n-26)."""
    from oracle import cpu
    wl = _workloads()

    threads = os.cpu_count() or 1
    spec = wl.hadamard_benchmark(n_s, iterations=1)
    if cpu.ref_available("f64"):
        r = cpu.RefDGM(n_s, "f64")
        r.set_memory_value(0)
        for steps, it, reset in spec.calls:
            r.set_function(steps, it, reset)
        r.tuning(cpu.RefDGM.T_PAR_CPU, thread_count=threads)
        t0 = time.perf_counter()
        r.execute(1)
        dt = time.perf_counter() - t0
        r.close()
        kind = "reference"
    else:
        from oracle import circuit_lang as cl

        ops = spec.build(cl.Circuit()).as_arrays()
        s0 = cpu.basis_state(n_s, 0)
        t0 = time.perf_counter()
        cpu.run_regions(s0, n_s, ops, threads=threads)
        dt = time.perf_counter() - t0
        kind = "port"
    per = dt * (1 << (n - n_s))
    return {"value": round(1.0 / per, 6), "unit": "layers/s", "cores": threads, "kind": kind,
            "sample": f"the layer at {n_s} qubits FP64 t_PAR_CPU ({dt:.2f} s), scaled x{1 << (n - n_s)} to {n} qubits"}


# ---------------------------------------------------------------------------
# Grover search (config 2): 26 qubits FP64, marked index 42
# ---------------------------------------------------------------------------

GROVER_N, GROVER_MARK, GROVER_STEP_ITERS = 26, 42, 64


def grover_parts(sq, n, mark):
    """The Grover circuit as two plans: H on every qubit, and one iteration
    (phase oracle on |mark>, H^n, sign flip on |0..0>, H^n)."""
    wl = _workloads()

    spec = wl.grover_search(n, mark)
    (h_steps, _, _), (it_steps, _, _) = spec.calls
    init, one = sq.Circuit(), sq.Circuit()
    for c in (init, one):
        for name, m in spec.gates.items():
            c.add_gate(name, np.asarray(m, dtype=np.complex128))
    init.set_function(h_steps, 1, True)
    one.set_function(it_steps, 1, False)
    return spec, init, one


def workload_grover(args, dist, sq):
    n, mark = args.qubits or GROVER_N, GROVER_MARK
    prec = args.precision
    spec, c_init, c_one = grover_parts(sq, n, mark)
    total_iters = spec.meta["iterations"]
    p_init, p_one = sq.Plan(c_init, n, prec), sq.Plan(c_one, n, prec)
    st = sq.State(n, prec).set_basis(0).execute(p_init)
    step_iters = GROVER_STEP_ITERS

    def step():
        st.execute(p_one, step_iters)

    with ClockSampler(dist.local_rank) as clk:
        ms, launches = run_timed(dist, sq, step, args.steps, args.warmup)
    ms_step = dist.max(ms / args.steps)
    value = dist.world * step_iters / (ms_step * 1e-3)
    stats = p_one.stats()
    S = st.nbytes
    passes_per_step = stats["passes"] * step_iters
    achieved = passes_per_step * 2 * S / (ms_step * 1e-3) / 1e9
    # outside the timed region: finish the search and check the answer
    done = (args.warmup + args.steps) * step_iters
    st.set_basis(0).execute(p_init).execute(p_one, total_iters)
    found, pmax = st.marginal_argmax((1 << n) - 1)
    st.free()
    peak, peak_kind = hbm_peak()
    line = base_line(args, dist, METRICS["grover"], value, "iterations/s", ms_step, prec, config_for(args))
    line["plan"] = {"passes_per_iteration": stats["passes"]}
    line["search"] = {"iterations": total_iters, "argmax": int(found), "probability": round(pmax, 12),
                      "ok": bool(found == mark and pmax > 0.99), "timed_iterations_before_check": done}
    line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4),
                        "traffic": round(TRAFFIC_OVER_ALGO[prec] * 2 * S / 1e9, 3), "traffic_unit": "GB per launch",
                        "traffic_source": "ncu capture of the 26-qubit %s layered case (same state size)" % prec.upper(),
                        "peak_source": peak_kind,
                        "kernel": "%s<%s,%d,%d>" % ("chain_kernel" if S <= (32 << 20) else "pass_kernel",
                                                    {"f64": "double", "f32": "float"}[prec], stats["reg_bits"],
                                                    stats["warp_bits"]),
                        "algorithmic_bytes_per_launch": 2 * S}
    line["gpu_launches"] = launches
    line["clocks"] = clk.summary()
    line["e2e"] = e2e_grover(dist, sq, c_init, c_one, n, step_iters) if not (args.skip_e2e or prec != "f64") else None
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_grover(args, n, mark)
    return line


def e2e_grover(dist, sq, c_init, c_one, n, iters):
    """One step through the reference's C-ABI: GpuExecutionWrapper with the PT list of one iteration and
    iterations = 64, on a host state (1 GiB each way)."""
    L = sq.load_dropin("f64")
    L.setDevice(dist.local_rank)
    host = np.zeros(1 << n, dtype=np.complex128)
    host[0] = 1.0
    L.GpuExecutionWrapper(host.ctypes.data, c_init.ref_pts("f64"), n, 4, 8, 1, 64, 2, 1)
    pts = c_one.ref_pts("f64")
    t0 = time.perf_counter()
    L.GpuExecutionWrapper(host.ctypes.data, pts, n, 4, 8, 1, 64, 2, iters)
    dt = dist.max(time.perf_counter() - t0)
    return {"value": round(dist.world * iters / dt, 4), "unit": "iterations/s", "h2d_bytes_per_step": int(host.nbytes),
            "d2h_bytes_per_step": int(host.nbytes), "path": "GpuExecutionWrapper (reference C-ABI), host state",
            "seconds": round(dt, 3)}


def cpu_baseline_grover(args, n, mark, n_s=22, iters=8):
    """t_PAR_CPU on a bounded sample: 8 iterations at 22 qubits, scaled by 2^(n-22)."""
    from oracle import cpu
    wl = _workloads()

    threads = os.cpu_count() or 1
    spec = wl.grover_search(n_s, mark, iterations=iters)
    if cpu.ref_available("f64"):
        r = cpu.RefDGM(n_s, "f64")
        for name, m in spec.gates.items():
            r.add_gate(name, m)
        r.set_memory_value(0)
        (h_steps, _, _), (it_steps, _, _) = spec.calls
        r.set_function(h_steps, 1, True)
        r.tuning(cpu.RefDGM.T_PAR_CPU, thread_count=threads)
        r.execute(1)
        r.set_function(it_steps, iters, False)
        t0 = time.perf_counter()
        r.execute(1)
        dt = time.perf_counter() - t0
        r.close()
        kind = "reference"
    else:
        from oracle import circuit_lang as cl

        ops = spec.build(cl.Circuit()).as_arrays()
        s0 = cpu.basis_state(n_s, 0)
        t0 = time.perf_counter()
        cpu.run_regions(s0, n_s, ops, threads=threads)
        dt = time.perf_counter() - t0
        kind = "port"
    per_iter = dt / iters * (1 << (n - n_s))
    return {"value": round(1.0 / per_iter, 6), "unit": "iterations/s", "cores": threads, "kind": kind,
            "sample": f"{iters} Grover iterations at {n_s} qubits FP64 t_PAR_CPU ({dt:.2f} s), scaled "
                      f"x{1 << (n - n_s)} to {n} qubits"}


# ---------------------------------------------------------------------------
# batched launch (config 4): 512 circuits of 10-22 qubits in one graph
# ---------------------------------------------------------------------------

def batched_specs(seed, count=512, lo=10, hi=22):
    """Half exact QFTs of random basis inputs, half 10-layer random Rz/Ry+CNOT circuits; qubits uniform."""
    wl = _workloads()

    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.integers(lo, hi + 1))
        if i % 2:
            specs.append(wl.qft(n, int(rng.integers(1 << n))))
        else:
            specs.append(wl.random_layered(n, 10, seed=seed * 10007 + i))
    return specs


def batched_one(args, dist, sq, specs, circuits, prec):
    b = sq.Batch(prec, 2)
    for spec, c in zip(specs, circuits):
        b.add(c, spec.qubits, spec.init_index)
    t0 = time.perf_counter()
    tune = b.autotune()
    tune_s = time.perf_counter() - t0
    size = b.size()
    inputs = sq.PinnedArray((len(specs),), np.int64)
    inputs.array[:] = [spec.init_index for spec in specs]
    b.set_inputs(inputs.array)

    def step():
        b.run()

    ms, launches = run_timed(dist, sq, step, args.steps, args.warmup)
    b.check()
    ms_step = dist.max(ms / args.steps)
    value = dist.world * len(specs) / (ms_step * 1e-3)
    peak, peak_kind = hbm_peak()
    achieved = size["pass_bytes"] / (ms_step * 1e-3) / 1e9
    out = {"value": round(value, 4), "unit": "circuits/s", "ms_per_step": round(ms_step, 4),
           "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                        "kernel": f"batch_kernel ({prec})", "algorithmic_bytes_per_launch": size["pass_bytes"]},
           "autotune": {**tune, "seconds": round(tune_s, 2)}, "tasks": size["tasks"], "tile_items": size["items"],
           "arena_bytes": size["arena_bytes"], "gpu_launches": launches}
    if not args.skip_e2e:
        # end to end: the step's initial basis indices from pinned host memory, the graph, and every final
        # state back into pinned host memory
        host = sq.PinnedArray((size["arena_bytes"],), np.uint8)
        for _ in range(2):
            b.set_inputs(inputs.array).run().download(host)
        sq.synchronize()
        dist.barrier()
        with sq.Timer() as t:
            for _ in range(args.steps):
                b.set_inputs(inputs.array).run().download(host)
        sq.synchronize()
        e_ms = dist.max(t.ms / args.steps)
        out["e2e"] = {"value": round(dist.world * len(specs) / (e_ms * 1e-3), 4), "unit": "circuits/s",
                      "h2d_bytes_per_step": int(inputs.nbytes), "d2h_bytes_per_step": int(size["arena_bytes"]),
                      "path": "hgm_batch_set_inputs (pinned) -> hgm_batch_run -> hgm_batch_download (pinned)"}
        del host
    del b
    return out


def plain_batched(sq, specs, circuits, prec, limit_s):
    """The same circuits one by one through the plain t_GPU drop-in (host state each), up to limit_s seconds."""
    L = sq.load_dropin(prec)
    L.setDevice(0)
    dt = np.complex128 if prec == "f64" else np.complex64
    done, t0 = 0, time.perf_counter()
    for spec, c in zip(specs, circuits):
        host = np.zeros(1 << spec.qubits, dtype=dt)
        host[spec.init_index] = 1.0
        L.GpuExecutionWrapper(host.ctypes.data, c.ref_pts(prec), spec.qubits, 4, 8, 1, 64, 2, 1)
        done += 1
        if time.perf_counter() - t0 > limit_s:
            break
    el = time.perf_counter() - t0
    return {"value": round(done / el, 4), "unit": "circuits/s", "circuits": done, "seconds": round(el, 3),
            "path": f"GpuExecutionWrapper {prec.upper()} (reference C-ABI), host state per circuit"}


def workload_batched(args, dist, sq):
    count = args.requests or 512
    specs = batched_specs(4242, count)
    circuits = [spec.build(sq.Circuit()) for spec in specs]
    with ClockSampler(dist.local_rank) as clk:
        f32 = batched_one(args, dist, sq, specs, circuits, "f32")
    f64 = batched_one(args, dist, sq, specs, circuits, "f64")
    line = base_line(args, dist, METRICS["batched"], f32["value"], "circuits/s", f32["ms_per_step"], "f32",
                     config_for(args))
    line["inputs"] = ("plans and basis indices uploaded before the timed region; a step is one graph replay "
                      "(state init + every circuit)")
    line["gpu_launches"] = f32["gpu_launches"]
    line["roofline"] = f32["roofline"]
    line["fp32"] = f32
    line["fp64"] = f64
    line["e2e"] = f32.get("e2e")
    line["clocks"] = clk.summary()
    if not args.skip_e2e:
        line["plain_fp32"] = plain_batched(sq, specs, circuits, "f32", args.plain_limit)
        line["plain_fp64"] = plain_batched(sq, specs, circuits, "f64", args.plain_limit)
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_batched(args, specs)
    return line


def gate_layers_hbm(sq, n, prec, peak, peak_kind, cases=("hadamard_layer", "random_layers_2")):
    """Short gate-layer measurements on one large state: one H layer on every qubit and two random Rz/Ry+CNOT
    layers, each timed once with CUDA events after one untimed run; per-pass HBM GB/s as a fraction of the
    peak (a pass reads and writes the state once)."""
    wl = _workloads()
    st = sq.State(n, prec).set_basis(0)
    S = st.nbytes
    out = {"qubits": n, "precision": prec, "state_bytes": S, "peak": peak, "peak_source": peak_kind}
    for name in cases:
        spec = wl.hadamard_benchmark(n, 1) if name == "hadamard_layer" else wl.random_layered(n, 2, seed=77)
        plan = sq.Plan(spec.build(sq.Circuit()), n, prec)
        st.execute(plan)
        sq.synchronize()
        with sq.Timer() as t:
            st.execute(plan)
        passes = plan.stats()["passes"]
        gbs = passes * 2 * S / (t.ms * 1e-3) / 1e9
        layers = 1 if name == "hadamard_layer" else 2
        out[name] = {"ms": round(t.ms, 3), "passes": passes, "layers_per_s": round(layers / (t.ms * 1e-3), 3),
                     "GB/s": round(gbs, 1), "frac": round(gbs / peak, 4)}
    norm = st.norm()
    out["norm_after"] = norm
    st.free()
    return out


def grover_check(sq, peak, peak_kind, n=GROVER_N, mark=GROVER_MARK):
    """The 26-qubit FP64 Grover search, short form: iterations/s over 3 timed steps of 64 iterations (after one
    untimed step), then the full 6433-iteration search with its argmax and probability."""
    spec, c_init, c_one = grover_parts(sq, n, mark)
    p_init, p_one = sq.Plan(c_init, n, "f64"), sq.Plan(c_one, n, "f64")
    st = sq.State(n, "f64").set_basis(0).execute(p_init)
    st.execute(p_one, GROVER_STEP_ITERS)
    sq.synchronize()
    with sq.Timer() as t:
        for _ in range(3):
            st.execute(p_one, GROVER_STEP_ITERS)
    iters_s = 3 * GROVER_STEP_ITERS / (t.ms * 1e-3)
    passes = p_one.stats()["passes"]
    gbs = passes * 2 * st.nbytes * iters_s / 1e9
    total = spec.meta["iterations"]
    with sq.Timer() as t2:
        st.set_basis(0).execute(p_init).execute(p_one, total)
    found, pmax = st.marginal_argmax((1 << n) - 1)
    st.free()
    return {"iterations_per_s": round(iters_s, 2), "passes_per_iteration": passes, "GB/s": round(gbs, 1),
            "frac": round(gbs / peak, 4), "peak_source": peak_kind, "full_search_s": round(t2.ms * 1e-3, 3),
            "iterations": total, "argmax": int(found), "probability": round(pmax, 12),
            "ok": bool(found == mark and pmax > 0.99)}


def batched_check(sq, peak, peak_kind):
    """The 512-circuit batch (10-22 qubits, half QFT, half 10-layer random circuits), autotuned, FP32 and FP64:
    circuits/s over 3 graph replays after one untimed replay."""
    specs = batched_specs(4242, 512)
    circuits = [spec.build(sq.Circuit()) for spec in specs]
    out = {}
    for prec in ("f32", "f64"):
        b = sq.Batch(prec, 2)
        for spec, c in zip(specs, circuits):
            b.add(c, spec.qubits, spec.init_index)
        tune = b.autotune()
        b.run()
        sq.synchronize()
        with sq.Timer() as t:
            for _ in range(3):
                b.run()
        b.check()
        size = b.size()
        ms = t.ms / 3
        gbs = size["pass_bytes"] / (ms * 1e-3) / 1e9
        out[prec] = {"circuits_per_s": round(512 / (ms * 1e-3), 1), "ms_per_run": round(ms, 3),
                     "GB/s": round(gbs, 1), "frac": round(gbs / peak, 4),
                     "autotune": {"warp_bits": tune["warp_bits"], "low_bits": tune["low_bits"]}}
        del b
    out["peak_source"] = peak_kind
    return out


def ref_run_request(spec, prec, threads, gpu=False):
    """Runs one circuit on the reference's own engine the way its algorithm libraries do
    (src/algorithms/lib_general.cpp:30-36, lib_grover.cpp:30-59): a DGM with its state allocated,
    setMemoryValue, the circuit's gates (Gates::addGate), one setFunction per call of the circuit and one
    execute -- on t_PAR_CPU with `threads` OpenMP threads, or with gpu=True on t_GPU, the reference's own
    kernel.cu built for sm_100a, with the CLIs' default GPU tuning (include/cli/cli_common.h:8-17).
    Returns the wall seconds of all of it."""
    from oracle import cpu

    t0 = time.perf_counter()
    r = cpu.RefDGM(spec.qubits, prec, gpu=gpu)
    r.set_memory_value(spec.init_index)
    spec.build(r)
    if gpu:
        r.tuning(cpu.RefDGM.T_GPU)
    else:
        r.tuning(cpu.RefDGM.T_PAR_CPU, thread_count=threads)
    r.execute(1)
    dt = time.perf_counter() - t0
    r.close()
    return dt


def ref_stream(specs, prec, threads, budget_s, cursor=0):
    """Runs specs[cursor], specs[cursor+1], ... unscaled on the reference until budget_s seconds have been
    spent (the request that crosses the budget completes); returns (requests run, seconds, per-request
    seconds, next cursor).  Wraps around the list."""
    done, spent, each = 0, 0.0, []
    while spent < budget_s and specs:
        dt = ref_run_request(specs[cursor % len(specs)], prec, threads)
        each.append(dt)
        spent += dt
        done += 1
        cursor += 1
    return done, spent, each, cursor


def cpu_baseline_batched(args, specs, budget_s=20.0):
    """The reference's t_PAR_CPU (FP32, unmodified) on the batch's circuits in order, each run unscaled and
    alone, for about budget_s seconds."""
    from oracle import cpu

    threads = os.cpu_count() or 1
    if not cpu.ref_available("f32"):
        return None
    done, spent, _, _ = ref_stream(specs, "f32", threads, budget_s)
    return {"value": round(done / spent, 6), "unit": "circuits/s", "cores": threads, "kind": "reference",
            "sample": (f"the first {done} of the {len(specs)} circuits in batch order" if done <= len(specs) else
                       f"{done} circuits: the {len(specs)} in batch order, then again from the first") +
                      f" on t_PAR_CPU FP32, each unscaled, one setFunction + execute per circuit ({spent:.1f} s)"}


# ---------------------------------------------------------------------------
# served stream (continuous batching)
# ---------------------------------------------------------------------------

SERVED_METRIC = "served circuits/s (FP32 continuous batching, 1-F<1e-6 vs FP64)"


def served_requests(seed, count, max_qubits=28):
    """The serving mix: 60% random layered (12-26 qubits, depth 20), 30% QFT
    (16-28 qubits) on a random basis input, 10% Grover (14-20 qubits, marked
    index uniform); all drawn from `seed`."""
    wl = _workloads()

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        u = rng.random()
        if u < 0.6:
            n = int(rng.integers(12, 27))
            spec, mask = wl.random_layered(min(n, max_qubits), 20, seed=seed * 100003 + i), 0
        elif u < 0.9:
            n = min(int(rng.integers(16, 29)), max_qubits)
            spec = wl.qft(n, int(rng.integers(1 << n)))
            mask = 0
        else:
            m = int(rng.integers(14, 21))
            spec = wl.grover_search(m, int(rng.integers(1 << m)))
            mask = (1 << m) - 1
        reqs.append((spec, mask))
    return reqs


def serve_step(sq, srv, reqs, items, rate_hz, rng, planned):
    """Submits `reqs` with Poisson arrivals at rate_hz (0 = all at once) and waits for every result.
    planned: items are device-resident plans (hgm_server_submit_plan); else host circuits that the server
    plans and uploads (hgm_server_submit)."""
    t0 = time.perf_counter()
    gaps = rng.exponential(1.0 / rate_hz, len(reqs)) if rate_hz > 0 else np.zeros(len(reqs))
    due = t0
    out = []
    for (spec, mask), item, gap in zip(reqs, items, gaps):
        due += gap
        while True:
            now = time.perf_counter()
            if now >= due:
                break
            out += srv.poll(wait_ms=0)
            time.sleep(min(0.0005, due - now))
        if planned:
            srv.submit_plan(item, spec.init_index, mask)
        else:
            srv.submit(item, spec.qubits, spec.init_index, mask)
    out += srv.drain(len(reqs) - len(out))
    return out, time.perf_counter() - t0


def served_run(args, dist, sq, srv, steps_reqs, steps_items, planned, rng, rate=None):
    """Warm-up steps, then the timed steps (device-timed with a synchronize on both sides); arrivals are
    Poisson at `rate` requests/s (default args.rate; 0 = all of a step at once)."""
    rate = args.rate if rate is None else rate
    for w in range(args.warmup):
        serve_step(sq, srv, steps_reqs[w], steps_items[w], 0, rng, planned)
    sq.synchronize()
    dist.barrier()
    lat, done = [], 0
    launches0 = sq.kernel_launches()
    with ClockSampler(dist.local_rank) as clk:
        with sq.Timer() as t:
            for s in range(args.steps):
                res, _ = serve_step(sq, srv, steps_reqs[args.warmup + s], steps_items[args.warmup + s],
                                    rate, rng, planned)
                lat += [r["latency_s"] for r in res]
                done += len(res)
                assert all(r["status"] == 0 for r in res)
            sq.synchronize()
    launches = sq.kernel_launches() - launches0
    dist.barrier()
    ms = dist.max(t.ms)
    lat = np.array(lat)
    latency = {"p50": round(float(np.percentile(lat, 50)) * 1e3, 3), "p99": round(float(np.percentile(lat, 99)) * 1e3, 3),
               "mean": round(float(lat.mean()) * 1e3, 3)}
    return dist.sum(done) / (ms * 1e-3), ms, latency, launches, clk.summary()


def workload_served(args, dist, sq):
    count = args.requests or 48
    steps_reqs = [served_requests(1000 + s, count) for s in range(args.warmup + args.steps)]
    steps_circuits = [[spec.build(sq.Circuit()) for spec, _ in reqs] for reqs in steps_reqs]
    # every request's plan, built and uploaded before any timed region: the device-resident inputs
    steps_plans = [[sq.Plan(c, spec.qubits, "f32").upload() for (spec, _), c in zip(reqs, cs)]
                   for reqs, cs in zip(steps_reqs, steps_circuits)]
    upload = [sum(p.stats()["upload_bytes"] for p in plans) for plans in steps_plans]
    srv = sq.Server("f32", budget_bytes=150 << 30, max_inflight=args.inflight, order=args.order)
    value, ms, latency, launches, clocks = served_run(args, dist, sq, srv, steps_reqs, steps_plans, True,
                                                      np.random.default_rng(7))
    ms_step = ms / args.steps
    # end to end: host circuits in (planned and uploaded by the server inside the timed region), results out
    e2e = None
    if not args.skip_e2e:
        v2, ms2, lat2, _, _ = served_run(args, dist, sq, srv, steps_reqs, steps_circuits, False,
                                         np.random.default_rng(7))
        timed = range(args.warmup, args.warmup + args.steps)
        e2e = {"value": round(v2, 4), "unit": "circuits/s",
               "h2d_bytes_per_step": int(round(np.mean([upload[s] for s in timed]))),
               "d2h_bytes_per_step": 32 * count,
               "path": "hgm_server_submit (host circuit: planned, op records uploaded) -> hgm_server_poll "
                       "(norm, argmax, pmax to host)",
               "latency_ms": lat2, "ms_per_step": round(ms2 / args.steps, 3)}
    # Poisson arrivals at fractions of the measured capacity: throughput and latency per offered rate
    sweep = []
    if not args.skip_sweep and args.rate == 0:
        for frac in (0.5, 0.8):
            rate = frac * value / dist.world
            v3, ms3, lat3, _, _ = served_run(args, dist, sq, srv, steps_reqs, steps_plans, True,
                                             np.random.default_rng(11), rate=rate)
            sweep.append({"offered_rate_hz": round(rate, 2), "fraction_of_capacity": frac,
                          "circuits_per_s": round(v3, 4), "latency_ms": lat3})
    srv.close()
    del steps_plans
    # fidelity of the FP32 served results against FP64 reruns (first timed step)
    fid = served_fidelity(sq, steps_reqs[args.warmup], steps_circuits[args.warmup]) if not args.skip_fidelity else None
    # the same requests one by one through the plain FP64 t_GPU drop-in (host states)
    plain = plain_fp64(sq, steps_reqs[args.warmup], steps_circuits[args.warmup], args.plain_limit) \
        if not args.skip_e2e else None
    peak, peak_kind = hbm_peak()
    line = base_line(args, dist, SERVED_METRIC, value, "circuits/s", ms_step, "f32", config_for(args))
    line["inputs"] = ("plans built and uploaded before the timed region (hgm_server_submit_plan); states "
                      "initialised on the device")
    line["latency_ms"] = latency
    line["rate_sweep"] = sweep
    line["fidelity"] = fid
    line["plain_fp64"] = plain
    line["gpu_launches"] = launches
    line["clocks"] = clocks
    line["roofline"] = served_roofline(sq, args, peak, peak_kind)
    if not args.skip_layers:
        line["gate_layers_30q_f64"] = gate_layers_hbm(sq, 30, "f64", peak, peak_kind)
        line["layered_32q_f32"] = gate_layers_hbm(sq, 32, "f32", peak, peak_kind, cases=("random_layers_2",))
        line["grover_26q_f64"] = grover_check(sq, peak, peak_kind)
        line["batched_512"] = batched_check(sq, peak, peak_kind)
    line["e2e"] = e2e
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_served(args, steps_reqs[args.warmup])
    return line


def served_fidelity(sq, reqs, circuits):
    worst_gap, worst_err = 0.0, 0.0
    for (spec, mask), c in zip(reqs, circuits):
        a = sq.State(spec.qubits, "f32").set_basis(spec.init_index)
        a.execute(sq.Plan(c, spec.qubits, "f32"))
        b = sq.State(spec.qubits, "f64").set_basis(spec.init_index)
        b.execute(sq.Plan(c, spec.qubits, "f64"))
        ov = b.inner(a)
        gap = 1.0 - abs(ov) ** 2 / (a.norm() * b.norm())
        worst_gap = max(worst_gap, gap)
        worst_err = max(worst_err, b.max_abs_diff(a))
        a.free()
        b.free()
    return {"max_1_minus_F": worst_gap, "max_abs_amp_err": worst_err, "requests": len(reqs),
            "ok": bool(worst_gap < 1e-6)}


def plain_fp64(sq, reqs, circuits, limit):
    """The same requests through GpuExecutionWrapper (FP64 drop-in), one by one, host state in and out."""
    L = sq.load_dropin("f64")
    L.setDevice(0)
    t0 = time.perf_counter()
    k = 0
    for (spec, mask), c in zip(reqs, circuits):
        host = np.zeros(1 << spec.qubits, dtype=np.complex128)
        host[spec.init_index] = 1.0
        L.GpuExecutionWrapper(host.ctypes.data, c.ref_pts("f64"), spec.qubits, 4, 8, 1, 64, 2, 1)
        k += 1
        if limit and time.perf_counter() - t0 > limit:
            break
    dt = time.perf_counter() - t0
    return {"value": round(k / dt, 4), "unit": "circuits/s", "requests": k, "seconds": round(dt, 3),
            "path": "GpuExecutionWrapper FP64 (reference C-ABI), host state per request"}


def served_roofline(sq, args, peak, peak_kind):
    """Roofline of the dominant kernel (the FP32 pass kernel) on the mix's largest layered circuit."""
    wl = _workloads()

    n = 26
    spec = wl.random_layered(n, 20, seed=99)
    plan = sq.Plan(spec.build(sq.Circuit()), n, "f32")
    st = sq.State(n, "f32").set_basis(0)
    st.execute(plan)
    sq.synchronize()
    with sq.Timer() as t:
        st.execute(plan)
    stats = plan.stats()
    S = st.nbytes
    st.free()
    achieved = stats["passes"] * 2 * S / (t.ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": round(TRAFFIC_OVER_ALGO["f32"] * 2 * S / 1e9, 3), "traffic_unit": "GB per launch",
            "traffic_source": "ncu capture of this 26-qubit FP32 layered case",
            "peak_source": peak_kind,
            "kernel": "pass_kernel<float,%d,%d>" % (stats["reg_bits"], stats["warp_bits"]),
            "case": f"{n}q FP32 random layered, 20 layers, {stats['passes']} passes",
            "algorithmic_bytes_per_launch": 2 * S}


def cpu_baseline_served(args, reqs, budget_s=20.0):
    """The reference's t_PAR_CPU (FP32, unmodified) on the served stream's requests in order, each run
    unscaled and alone (one setFunction + execute per request), for about budget_s seconds."""
    from oracle import cpu

    threads = os.cpu_count() or 1
    if not cpu.ref_available("f32"):
        return None
    specs = [spec for spec, _ in reqs][::4]
    done, spent, _, _ = ref_stream(specs, "f32", threads, budget_s)
    return {"value": round(done / spent, 6), "unit": "circuits/s", "cores": threads, "kind": "reference",
            "sample": f"every 4th request of the first timed step, the first {done} of them, on t_PAR_CPU FP32, "
                      f"each unscaled, one setFunction + execute per request ({spent:.1f} s)"}


WORKLOADS = {"layered": workload_layered, "served": workload_served, "grover": workload_grover,
             "batched": workload_batched, "hadamard": workload_hadamard, "qft": workload_qft}

METRICS = {"layered": "gate-layers/s (30q random Rz/Ry+CNOT layers)",
           "grover": "Grover iterations/s (marked index 42; 26q FP64 by default)",
           "hadamard": "gate-layers/s (H on every qubit, 30q FP64)",
           "batched": "batched circuits/s (512 circuits, 10-22 qubits, one persistent kernel)",
           "served": SERVED_METRIC,
           "qft": "QFT circuits/s (textbook QFT of a basis state)"}


def config_for(args):
    """The `config` of a workload's JSON line: what the workload is, identical in both arms (engine-side
    figures such as passes per step go in the line's `plan` key)."""
    w = args.workload
    if w == "served":
        count = args.requests or 48
        return {"workload": f"served-mix-{count}req", "requests_per_step": count, "rate_hz": args.rate,
                "max_inflight": args.inflight, "admission_order": args.order, "budget_bytes": 150 << 30,
                "precision": "fp32 amplitudes, fp64 gate matrices, norms and argmax",
                "mix": "60% layered 12-26q d20, 30% QFT 16-28q, 10% Grover 14-20q",
                "stream": "step s draws its requests from seed 1000 + s",
                "l2": "states up to 2 GiB; no flush (serving keeps states resident)"}
    if w == "batched":
        count = args.requests or 512
        return {"workload": f"batched-{count}", "circuits": count, "qubits": "uniform 10-22",
                "mix": "half QFT of a random basis input, half 10-layer random Rz/Ry+CNOT",
                "l2": "arena of all states (~2.6 GB FP32) > 126 MB L2, no flush needed"}
    if w == "layered":
        n, layers = args.qubits or 30, args.layers or 40
        S = (1 << n) * (16 if args.precision == "f64" else 8)
        return {"workload": f"layered-{n}q-{layers}layers", "qubits": n, "layers": layers,
                "precision": {"f64": "fp64", "f32": "fp32"}[args.precision], "state_bytes": S,
                "l2": f"state {S / 2**30:g} GiB > 126 MB L2, no flush needed"}
    if w == "hadamard":
        n = args.qubits or 30
        S = 16 << n
        return {"workload": f"hadamard-layer-{n}q-fp64", "qubits": n, "gates_per_layer": n, "state_bytes": S,
                "l2": f"state {S / 2**30:g} GiB > 126 MB L2, no flush needed"}
    if w == "qft":
        n = args.qubits or 28
        S = (1 << n) * (16 if args.precision == "f64" else 8)
        return {"workload": f"qft-{n}q", "qubits": n, "precision": {"f64": "fp64", "f32": "fp32"}[args.precision],
                "state_bytes": S, "l2": f"state {S / 2**30:g} GiB > 126 MB L2, no flush needed"}
    if w == "grover":
        n = args.qubits or GROVER_N
        S = (1 << n) * (16 if args.precision == "f64" else 8)
        l2 = (f"state {S / 2**30:g} GiB > 126 MB L2, no flush needed" if S > (126 << 20) else
              f"state {S / 2**20:g} MiB stays in L2 (its passes run chained); no flush")
        return {"workload": f"grover-{n}q-{'fp64' if args.precision == 'f64' else 'fp32'}", "qubits": n,
                "marked": GROVER_MARK, "iterations_per_step": GROVER_STEP_ITERS, "state_bytes": S, "l2": l2}
    return {"workload": w}


def base_line(args, dist, metric, value, unit, ms_step, dtype, config):
    return {"metric": metric, "value": round(value, 4), "unit": unit, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)", "config": config}


def reference_stream_specs(args):
    """The circuits of the workload as a stream, in the order the repo arm's timed steps run them."""
    if args.workload == "served":
        count = args.requests or 48
        return [spec for s in range(args.warmup, args.warmup + args.steps + 4)
                for spec, _ in served_requests(1000 + s, count)], "f32"
    if args.workload == "batched":
        return batched_specs(4242, args.requests or 512), "f32"
    return None, None


def reference_gpu_leg(args):
    """The reference's own t_GPU (kernel.cu for sm_100a, FP32, oracle/_ref/libref_gpu_f32.so) on the first
    timed step's requests in order, each unscaled, for about args.ref_gpu_s seconds after one untimed
    request.  Runs in a child process (`--impl reference-gpu`): the reference exits the process on any CUDA
    error (src/core/kernel.cu:439-447)."""
    from oracle import cpu

    if not cpu.ref_available("f32", gpu=True):
        return {"unavailable": "the reference's GPU backend (oracle/_ref/libref_gpu_f32.so) was not built"}
    count = args.requests or 48
    specs = [spec for spec, _ in served_requests(1000 + args.warmup, count)]
    small = min(specs, key=lambda s: (s.qubits, s.n_ops_estimate()))
    ref_run_request(small, "f32", 1, gpu=True)  # CUDA context and module load
    done, spent, each = 0, 0.0, []
    for spec in specs:
        dt = ref_run_request(spec, "f32", 1, gpu=True)
        each.append(dt)
        spent += dt
        done += 1
        if spent >= args.ref_gpu_s:
            break
    return {"value": round(done / spent, 4), "unit": "circuits/s", "requests": done, "seconds": round(spent, 3),
            "latency_ms": {"p50": round(float(np.percentile(each, 50)) * 1e3, 3),
                           "p99": round(float(np.percentile(each, 99)) * 1e3, 3)},
            "path": "the reference's DGM on t_GPU (GpuExecutionWrapper of its kernel.cu, built for sm_100a with "
                    "max_target_bit initialised), default GPU tuning, host state per request",
            "sample": f"the first {done} requests of the first timed step, in order, each unscaled"}


def reference_gpu_in_child(args):
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference-gpu", "--requests", str(args.requests or 48),
           "--warmup", str(args.warmup), "--ref-gpu-s", str(args.ref_gpu_s)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR",
                                                                "MASTER_PORT")}
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=args.ref_gpu_s * 4 + 120, env=env)
        lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
        if p.returncode == 0 and lines:
            return json.loads(lines[-1])
        return {"unavailable": f"child exited {p.returncode}: {(p.stdout + p.stderr).strip()[-300:]}"}
    except Exception as e:
        return {"unavailable": f"{type(e).__name__}: {e}"}


def reference_arm(args, dist):
    """The reference's own CPU implementation (t_PAR_CPU, oracle/_ref), rank 0 only, with every host thread.

    served / batched: each step runs the workload's circuits in stream order, unscaled, one setFunction +
    execute per circuit as the reference's libraries do, until args.ref_step_s seconds have been spent (the
    circuit that crosses the budget completes); value = circuits run / seconds.  The other workloads time
    their bounded, scaled samples (cpu_baseline_*), each a single setFunction + execute."""
    if dist.rank != 0:
        return None
    from oracle import cpu

    threads = os.cpu_count() or 1
    specs, prec = reference_stream_specs(args)
    line = {"metric": METRICS.get(args.workload, args.workload), "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "impl": "reference", "data": "synthetic (seeded)", "config": config_for(args)}
    if specs is not None:
        if not cpu.ref_available(prec):
            return {"impl": "reference", "unavailable": "the reference engine (oracle/_ref) was not built"}
        small = min(specs, key=lambda s: (s.qubits, s.n_ops_estimate()))
        for _ in range(args.warmup):
            ref_run_request(small, prec, threads)
        done, spent, each, cursor = 0, 0.0, [], 0
        for _ in range(args.steps):
            d, s, e, cursor = ref_stream(specs, prec, threads, args.ref_step_s, cursor)
            done, spent, each = done + d, spent + s, each + e
        v = done / spent
        unit = "circuits/s"
        sample = (f"the first {done} circuits of the stream (the timed steps' circuits in order), each unscaled, "
                  f"one setFunction + execute per circuit on t_PAR_CPU {prec.upper()} "
                  f"({args.steps} steps of >= {args.ref_step_s:g} s, {spent:.1f} s in all)")
        line.update({"value": round(v, 6), "unit": unit, "ms_per_step": round(spent / args.steps * 1e3, 3),
                     "dtype": prec, "circuits_run": done,
                     "latency_ms": {"p50": round(float(np.percentile(each, 50)) * 1e3, 3),
                                    "p99": round(float(np.percentile(each, 99)) * 1e3, 3),
                                    "note": "each circuit's run time alone (sequential, no queueing)"}})
    else:
        fn = {"layered": cpu_baseline_layered,
              "grover": lambda a: cpu_baseline_grover(a, a.qubits or GROVER_N, GROVER_MARK),
              "hadamard": lambda a: cpu_baseline_hadamard(a, a.qubits or 30)}.get(args.workload)
        if fn is None:
            return {"impl": "reference", "unavailable": f"no reference timing for workload {args.workload}"}
        for _ in range(args.warmup):
            fn(args)
        t0 = time.perf_counter()
        vals = [fn(args) for _ in range(max(1, args.steps))]
        wall = time.perf_counter() - t0
        v = statistics.median([x["value"] for x in vals])
        unit, sample = vals[0]["unit"], vals[0]["sample"]
        line.update({"value": v, "unit": unit, "ms_per_step": round(wall / max(1, args.steps) * 1e3, 3),
                     "dtype": "f64"})
    line["cpu_baseline"] = {"value": line["value"], "unit": unit, "cores": threads, "kind": "reference",
                            "sample": sample}
    if args.workload == "served" and not args.skip_ref_gpu:
        line["reference_gpu"] = reference_gpu_in_child(args)
    line["e2e"] = {"value": line["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 20 for served, whose 48-request steps last ~0.2 s; else 5)")
    ap.add_argument("--warmup", type=int, default=None, help="untimed warm-up steps (default 5 served, else 3)")
    ap.add_argument("--workload", default="served", choices=sorted(WORKLOADS))
    ap.add_argument("--requests", type=int, default=0, help="requests per served step (default 48)")
    ap.add_argument("--rate", type=float, default=0.0, help="Poisson arrival rate in requests/s (0: all at once)")
    ap.add_argument("--inflight", type=int, default=32, help="server slots")
    ap.add_argument("--order", default="arrival", choices=["arrival", "work_first"],
                    help="server admission order of queued requests")
    ap.add_argument("--plain-limit", type=float, default=60.0, help="seconds cap for the plain FP64 comparison")
    ap.add_argument("--skip-fidelity", action="store_true")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu"])
    ap.add_argument("--ref-gpu-s", type=float, default=30.0,
                    help="reference arm, served: seconds of the reference's own t_GPU leg")
    ap.add_argument("--skip-ref-gpu", action="store_true", help="reference arm: no t_GPU leg")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-sweep", action="store_true", help="served: no Poisson rate sweep")
    ap.add_argument("--skip-layers", action="store_true",
                    help="served: none of the other configurations' short measurements (30-qubit FP64 gate layers, "
                         "32-qubit FP32 layers, 26-qubit Grover, the 512-circuit batch)")
    ap.add_argument("--qubits", type=int, default=0, help="override the workload's qubit count (profiling runs)")
    ap.add_argument("--layers", type=int, default=0, help="override the layered workload's depth (profiling runs)")
    ap.add_argument("--precision", default=None, choices=["f64", "f32"],
                    help="layered / qft amplitude type (default f64 layered, f32 qft)")
    ap.add_argument("--ref-step-s", type=float, default=5.0,
                    help="reference arm, served/batched: seconds of reference work per step")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.workload == "served" else 5
    if args.warmup is None:
        args.warmup = 5 if args.workload == "served" else 3
    if args.precision is None:
        args.precision = "f32" if args.workload == "qft" else "f64"
    dist = Dist()
    try:
        if args.impl == "reference":
            line = reference_arm(args, dist)
        elif args.impl == "reference-gpu":
            line = reference_gpu_leg(args) if dist.rank == 0 else None
        else:
            import simulador_quantico_b200 as sq

            sq.init(dist.local_rank)
            line = WORKLOADS[args.workload](args, dist, sq)
        if dist.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
