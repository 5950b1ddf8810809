"""ctypes bindings to libhgm_b200.so (include/hgm_b200.h).

The shared library is built in-tree (simulador_quantico_b200/build.py) and
loaded from simulador_quantico_b200/lib/.  There is no fallback: if the
library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
ENGINE = LIB_DIR / "libhgm_b200.so"
DROPIN = {"f32": LIB_DIR / "libhgm_dropin_f32.so", "f64": LIB_DIR / "libhgm_dropin_f64.so"}

HGM_OK = 0
HGM_F64, HGM_F32 = 0, 1
HGM_ORDER_ARRIVAL, HGM_ORDER_WORK_FIRST = 0, 1
ERRORS = {1: "invalid", 2: "cuda", 3: "nomem", 4: "unsupported", 5: "timeout", 6: "busy"}


class HgmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hgm error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class ServerOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("budget_bytes", C.c_int64), ("max_inflight", C.c_int),
                ("keep_states", C.c_int), ("warp_bits", C.c_int), ("order", C.c_int)]


class Result(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int), ("qubits", C.c_int), ("latency_s", C.c_double),
                ("queue_s", C.c_double), ("exec_s", C.c_double), ("norm", C.c_double), ("argmax", C.c_int64),
                ("pmax", C.c_double)]


class PlanOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("warp_bits", C.c_int), ("low_bits", C.c_int), ("fuse", C.c_int),
                ("window", C.c_int), ("renorm_every", C.c_int), ("chained", C.c_int),
                ("split_layers", C.c_int), ("reg_bits", C.c_int)]


def _load():
    if not ENGINE.exists():
        raise ImportError(f"{ENGINE} is missing: build it with `python simulador_quantico_b200/build.py`")
    L = C.CDLL(str(ENGINE))
    vp, i, i64, d = C.c_void_p, C.c_int, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "hgm_last_error": ([], C.c_char_p),
        "hgm_init": ([i], i),
        "hgm_synchronize": ([], i),
        "hgm_mem_info": ([P(i64), P(i64)], i),
        "hgm_kernel_launches": ([], i64),
        "hgm_circuit_new": ([], vp),
        "hgm_circuit_free": ([vp], None),
        "hgm_circuit_add_gate": ([vp, C.c_char_p, P(d)], i),
        "hgm_circuit_set_function": ([vp, C.c_char_p, i, i], i),
        "hgm_circuit_append_op": ([vp, i, i64, i64, P(d)], i),
        "hgm_circuit_qubits": ([vp], i),
        "hgm_circuit_num_ops": ([vp], i64),
        "hgm_circuit_get_ops": ([vp, P(C.c_int32), P(i64), P(i64), P(d)], i),
        "hgm_circuit_ref_pts": ([vp, i], vp),
        "hgm_plan_default_opts": ([P(PlanOpts), i], None),
        "hgm_plan_create": ([vp, i, P(PlanOpts), P(vp)], i),
        "hgm_plan_create_from_ref_pts": ([vp, i, i, P(PlanOpts), P(vp)], i),
        "hgm_plan_free": ([vp], None),
        "hgm_plan_stats": ([vp, P(i64), P(i64), P(i64), P(i64)], i),
        "hgm_plan_upload": ([vp], i),
        "hgm_plan_export": ([vp, P(vp), P(i64), P(vp), P(i64), P(vp), P(i64), P(i), P(i)], i),
        "hgm_plan_layouts": ([vp, P(vp), P(i64)], i),
        "hgm_state_create": ([i, i, P(vp)], i),
        "hgm_state_free": ([vp], None),
        "hgm_state_qubits": ([vp], i),
        "hgm_state_precision": ([vp], i),
        "hgm_state_device_ptr": ([vp], vp),
        "hgm_state_set_basis": ([vp, i64], i),
        "hgm_state_upload": ([vp, vp, i64], i),
        "hgm_state_download": ([vp, vp, i64], i),
        "hgm_execute": ([vp, vp, i, vp], i),
        "hgm_plan_status": ([vp], i),
        "hgm_norm": ([vp, P(d)], i),
        "hgm_prob_one": ([vp, i, P(d)], i),
        "hgm_measure_qubit": ([vp, i, d, P(i), P(d)], i),
        "hgm_collapse_qubit": ([vp, i, i, P(d)], i),
        "hgm_marginal_probs": ([vp, C.c_uint64, P(d), i64], i),
        "hgm_marginal_argmax": ([vp, C.c_uint64, P(i64), P(d)], i),
        "hgm_inner": ([vp, vp, P(d), P(d)], i),
        "hgm_max_abs_diff": ([vp, vp, P(d)], i),
        "hgm_scale": ([vp, d], i),
        "hgm_norm_noalloc": ([vp, i, i, vp, vp], i),
        "hgm_batch_create": ([i, i, P(vp)], i),
        "hgm_batch_free": ([vp], None),
        "hgm_batch_add": ([vp, vp, i, i64, P(i)], i),
        "hgm_batch_finalize": ([vp], i),
        "hgm_batch_run": ([vp, vp], i),
        "hgm_batch_autotune": ([vp, vp, P(i), P(i), P(C.c_double)], i),
        "hgm_batch_set_inputs": ([vp, P(i64), vp], i),
        "hgm_batch_download": ([vp, vp, i64, vp], i),
        "hgm_pinned_alloc": ([i64, P(vp)], i),
        "hgm_pinned_free": ([vp], None),
        "hgm_batch_check": ([vp], i),
        "hgm_batch_inject_stall": ([vp, i, i64], i),
        "hgm_batch_size": ([vp, P(i), P(i64), P(i64), P(i64), P(i64)], i),
        "hgm_batch_state": ([vp, i], vp),
        "hgm_server_default_opts": ([P(ServerOpts), i], None),
        "hgm_server_create": ([P(ServerOpts), P(vp)], i),
        "hgm_server_free": ([vp], None),
        "hgm_server_submit": ([vp, vp, i, i64, C.c_uint64, P(i64)], i),
        "hgm_server_submit_plan": ([vp, vp, i64, C.c_uint64, P(i64)], i),
        "hgm_server_poll": ([vp, P(Result), i, P(i), i], i),
        "hgm_server_pending": ([vp, P(i), P(i), P(i64)], i),
        "hgm_server_result_state": ([vp, i64], vp),
        "hgm_server_release": ([vp, i64], i),
        "hgm_timer_start": ([], i),
        "hgm_timer_stop": ([P(d)], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


lib = _load()


def last_error() -> str:
    msg = lib.hgm_last_error()
    return msg.decode() if msg else ""


def check(rc: int):
    if rc != HGM_OK:
        raise HgmError(rc, last_error())
    return rc


def load_dropin(prec: str):
    """The reference-ABI library (setDevice / GpuExecutionWrapper / ...)."""
    so = DROPIN[prec]
    if not so.exists():
        raise ImportError(f"{so} is missing: build it with `python simulador_quantico_b200/build.py`")
    L = C.CDLL(str(so))
    L.setDevice.argtypes = [C.c_int]
    L.setDevice.restype = C.c_bool
    L.GpuExecutionWrapper.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 7
    L.GpuExecutionWrapper.restype = C.c_void_p
    L.ProjectState.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_long, C.c_long, C.c_int]
    L.ProjectState.restype = C.c_bool
    L.GetState.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_long, C.c_long, C.c_int]
    L.GetState.restype = C.c_bool
    return L
