"""Benchmark for the B200 state-vector engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

Workloads (synthetic, seeded; see DESIGN.md for the shapes):
  served   the serving stream: a seeded request mix (random layered
           circuits, QFTs, Grover searches) served by the continuous-batching
           server in FP32 with FP64 norm checks; metric served circuits/s
  layered  a 30-qubit, 40-layer random Rz/Ry + CNOT circuit in FP64; metric
           gate-layers/s (one step = the whole circuit)
  grover   Grover search as grover.out runs it (27 qubits incl. the ancilla,
           FP64); metric Grover iterations/s (one step = 64 iterations)

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

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


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
    from simulador_quantico_b200 import workloads as wl

    n, layers, prec = args.qubits or 30, args.layers or 40, "f64"
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
    # end to end through the reference's C-ABI with host buffers (1 step)
    e2e = e2e_layered(dist, sq, spec, n, prec) if not args.skip_e2e else None
    st.free()
    line = base_line(args, dist, "gate-layers/s (30q random Rz/Ry+CNOT layers)", value, "layers/s", ms_step,
                     "f64", {"workload": f"layered-{n}q-{layers}layers", "qubits": n, "layers": layers, "precision": "fp64",
                             "state_bytes": S, "passes_per_step": stats["passes"], "ops_after_fusion": stats["ops"],
                             "l2": "state 16 GiB >> 126 MB L2, no flush needed"})
    line["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                        "kernel": "pass_kernel<double,%d,%d>" % (stats["reg_bits"], stats["warp_bits"]),
                        "algorithmic_bytes_per_launch": 2 * S}
    line["gpu_launches"] = launches
    line["clocks"] = clk.summary()
    line["e2e"] = e2e
    if dist.rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline_layered(args)
    return line


def e2e_layered(dist, sq, spec, n, prec):
    L = sq.load_dropin(prec)
    L.setDevice(dist.local_rank)
    c = spec.build(sq.Circuit())
    pts = c.ref_pts(prec)
    host = np.zeros(1 << n, dtype=np.complex128)
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
    from simulador_quantico_b200 import workloads as wl

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


WORKLOADS = {"layered": workload_layered}


def base_line(args, dist, metric, value, unit, ms_step, dtype, config):
    return {"metric": metric, "value": round(value, 4), "unit": unit, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)", "config": config}


def reference_arm(args, dist):
    """The reference's own CPU implementation (t_PAR_CPU), rank 0 only."""
    if dist.rank != 0:
        return None
    fn = {"layered": cpu_baseline_layered}.get(args.workload)
    if fn is None:
        return {"impl": "reference", "unavailable": f"no reference timing for workload {args.workload}"}
    vals = []
    for _ in range(max(1, args.steps)):
        vals.append(fn(args))
    v = statistics.median([x["value"] for x in vals])
    first = vals[0]
    line = {"metric": args.metric_name, "value": v, "unit": first["unit"], "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "impl": "reference", "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": args.workload},
            "cpu_baseline": {"value": v, "unit": first["unit"], "cores": first["cores"], "kind": first["kind"],
                             "sample": first["sample"]},
            "e2e": {"value": v, "unit": first["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="layered", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--qubits", type=int, default=0, help="override the workload's qubit count (profiling runs)")
    ap.add_argument("--layers", type=int, default=0, help="override the layered workload's depth (profiling runs)")
    args = ap.parse_args()
    args.metric_name = {"layered": "gate-layers/s (30q random Rz/Ry+CNOT layers)"}.get(args.workload, args.workload)
    dist = Dist()
    try:
        if args.impl == "reference":
            line = reference_arm(args, dist)
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
