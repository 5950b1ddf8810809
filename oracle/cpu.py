"""ctypes bindings to the oracle's C restatement and the built reference.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

``run_serial`` / ``run_regions`` call oracle/_build/libsv_oracle.so (the C
restatement of DGM::CpuExecution1 and PCpuExecution1, oracle/sv_oracle.c).
``RefDGM`` drives the reference's own DGM class through
oracle/_ref/libref_{f32,f64}.so (oracle/ref_harness.cpp), built from the
reference sources by oracle/build_ref.sh; it is only available where that
library was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REF = HERE / "_ref"


class OracleOp(C.Structure):
    _fields_ = [
        ("target", C.c_int32),
        ("pad", C.c_int32),
        ("cmask", C.c_int64),
        ("cval", C.c_int64),
        ("m", C.c_double * 8),
    ]


_lib = None


def build():
    """Compile oracle/sv_oracle.c (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        so = BUILD / "libsv_oracle.so"
        if not so.exists():
            build()
        _lib = C.CDLL(str(so))
        for prec, real in (("f64", C.c_double), ("f32", C.c_float)):
            f = getattr(_lib, f"oracle_serial_{prec}")
            f.argtypes = [C.POINTER(real), C.c_int, C.POINTER(OracleOp), C.c_long, C.c_int]
            f.restype = None
            f = getattr(_lib, f"oracle_regions_{prec}")
            f.argtypes = [C.POINTER(real), C.c_int, C.POINTER(OracleOp), C.c_long, C.c_int,
                          C.c_int, C.c_int, C.c_int]
            f.restype = None
            f = getattr(_lib, f"oracle_norm_{prec}")
            f.argtypes = [C.POINTER(real), C.c_int]
            f.restype = C.c_double
            f = getattr(_lib, f"oracle_prob_one_{prec}")
            f.argtypes = [C.POINTER(real), C.c_int, C.c_int]
            f.restype = C.c_double
    return _lib


def pack_ops(target, cmask, cval, mat):
    """(target[], cmask[], cval[], mat[n,4] complex) -> OracleOp array."""
    n = len(target)
    arr = (OracleOp * max(n, 1))()
    m = np.asarray(mat, dtype=np.complex128).reshape(n, 4)
    mr = np.empty((n, 8), dtype=np.float64)
    mr[:, 0::2] = m.real
    mr[:, 1::2] = m.imag
    for i in range(n):
        o = arr[i]
        o.target = int(target[i])
        o.cmask = int(cmask[i])
        o.cval = int(cval[i])
        for k in range(8):
            o.m[k] = mr[i, k]
    return arr, n


def _state_buffer(state, prec):
    dt = np.float64 if prec == "f64" else np.float32
    s = np.ascontiguousarray(np.asarray(state, dtype=np.complex128 if prec == "f64" else np.complex64))
    buf = s.view(dt).copy()
    return buf


def run_serial(state, qubits, ops, iterations=1, prec="f64"):
    """DGM::CpuExecution1 restated (dgm_cpu_exec.cpp:11-35). Returns a new state."""
    buf = _state_buffer(state, prec)
    arr, n = ops if isinstance(ops, tuple) and len(ops) == 2 else pack_ops(*ops)
    real = C.c_double if prec == "f64" else C.c_float
    getattr(lib(), f"oracle_serial_{prec}")(buf.ctypes.data_as(C.POINTER(real)), qubits, arr, n, iterations)
    return buf.view(np.complex128 if prec == "f64" else np.complex64)


def run_regions(state, qubits, ops, iterations=1, prec="f64", threads=None, coalesced_bits=11, region_bits=14):
    """PCpuExecution1 restated (dgm_par_exec.cpp:82-132), OpenMP threads."""
    buf = _state_buffer(state, prec)
    arr, n = ops if isinstance(ops, tuple) and len(ops) == 2 else pack_ops(*ops)
    real = C.c_double if prec == "f64" else C.c_float
    threads = threads or os.cpu_count() or 1
    getattr(lib(), f"oracle_regions_{prec}")(buf.ctypes.data_as(C.POINTER(real)), qubits, arr, n, iterations,
                                            threads, coalesced_bits, region_bits)
    return buf.view(np.complex128 if prec == "f64" else np.complex64)


def basis_state(qubits, index, dtype=np.complex128):
    s = np.zeros(1 << qubits, dtype=dtype)
    s[index] = 1.0
    return s


# ---- the reference's own engine (built by oracle/build_ref.sh) ----------

def _ref_lib_name(prec, dropin=False, gpu=False):
    if gpu:
        return f"libref_gpu_{prec}.so"
    return f"libref_dropin_{prec}.so" if dropin else f"libref_{prec}.so"


def ref_available(prec="f64", dropin=False, gpu=False):
    """dropin: the reference's objects linked against the product's drop-in;
    gpu: linked with the reference's own GPU backend (kernel.cu, FP32 only)."""
    return (REF / _ref_lib_name(prec, dropin, gpu)).exists()


class RefDGM:
    """The reference's DGM (include/core/dgm.h:65-163) through ref_harness.cpp."""

    T_CPU, T_PAR_CPU, T_GPU, T_HYBRID = 0, 1, 2, 3
    _libs: dict = {}

    def __init__(self, qubits, prec="f64", dropin=False, gpu=False):
        self.lib = self._load(prec, dropin, gpu)
        self.qubits = qubits
        self.prec = prec
        self.h = self.lib.ref_dgm_new(qubits)

    @classmethod
    def _load(cls, prec, dropin, gpu=False):
        key = (prec, dropin, gpu)
        if key not in cls._libs:
            L = C.CDLL(str(REF / _ref_lib_name(prec, dropin, gpu)))
            L.ref_dgm_new.restype = C.c_void_p
            L.ref_dgm_new.argtypes = [C.c_int]
            L.ref_dgm_free.argtypes = [C.c_void_p]
            L.ref_dgm_set_tuning.argtypes = [C.c_void_p] + [C.c_int] * 9
            L.ref_dgm_add_gate.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
            L.ref_dgm_set_memory_value.argtypes = [C.c_void_p, C.c_long]
            L.ref_dgm_set_state.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
            L.ref_dgm_get_state.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
            L.ref_dgm_set_function.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int]
            L.ref_dgm_num_pts.argtypes = [C.c_void_p]
            L.ref_dgm_num_pts.restype = C.c_long
            L.ref_dgm_dump_pts.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                           C.POINTER(C.c_int64), C.POINTER(C.c_double)]
            L.ref_dgm_execute.argtypes = [C.c_void_p, C.c_int]
            L.ref_dgm_measure.argtypes = [C.c_void_p, C.c_int]
            L.ref_dgm_measure.restype = C.c_int
            L.ref_seed_rng.argtypes = [C.c_ulong]
            L.ref_uniform_sample.argtypes = [C.c_ulong]
            L.ref_uniform_sample.restype = C.c_double
            L.ref_dgm_colapse.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.ref_dgm_measure_many.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_long),
                                               C.POINTER(C.c_double), C.c_long]
            L.ref_dgm_measure_many.restype = C.c_long
            cls._libs[key] = L
        return cls._libs[key]

    def close(self):
        if self.h:
            self.lib.ref_dgm_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self, exec_type, thread_count=1, cpu_region_bits=14, cpu_coalesced_bits=11, gpu_count=1,
               gpu_region_bits=8, gpu_coalesced_bits=4, block_size=64, repeat_count=2):
        self.lib.ref_dgm_set_tuning(self.h, exec_type, thread_count, cpu_region_bits, cpu_coalesced_bits,
                                    gpu_count, gpu_region_bits, gpu_coalesced_bits, block_size, repeat_count)

    def add_gate(self, name, m):
        m = np.asarray(m, dtype=np.complex128).reshape(4)
        buf = np.empty(8, dtype=np.float64)
        buf[0::2], buf[1::2] = m.real, m.imag
        return bool(self.lib.ref_dgm_add_gate(self.h, name.encode(), buf.ctypes.data_as(C.POINTER(C.c_double))))

    def set_memory_value(self, pos):
        self.lib.ref_dgm_set_memory_value(self.h, pos)

    def set_state(self, state):
        buf = np.ascontiguousarray(np.asarray(state, dtype=np.complex128)).view(np.float64)
        self.lib.ref_dgm_set_state(self.h, buf.ctypes.data_as(C.POINTER(C.c_double)))

    def state(self):
        buf = np.empty(2 << self.qubits, dtype=np.float64)
        self.lib.ref_dgm_get_state(self.h, buf.ctypes.data_as(C.POINTER(C.c_double)))
        return buf.view(np.complex128)

    def set_function(self, steps, iterations=1, reset=True):
        if not isinstance(steps, str):
            steps = ";".join(steps)
        self.lib.ref_dgm_set_function(self.h, steps.encode(), iterations, 1 if reset else 0)

    def pts(self):
        n = self.lib.ref_dgm_num_pts(self.h)
        t = np.empty(n, np.int32)
        cm = np.empty(n, np.int64)
        cv = np.empty(n, np.int64)
        m = np.empty(n * 8, np.float64)
        if n:
            self.lib.ref_dgm_dump_pts(self.h, t.ctypes.data_as(C.POINTER(C.c_int32)),
                                      cm.ctypes.data_as(C.POINTER(C.c_int64)),
                                      cv.ctypes.data_as(C.POINTER(C.c_int64)),
                                      m.ctypes.data_as(C.POINTER(C.c_double)))
        mat = m.reshape(n, 4, 2)
        return t, cm, cv, mat[..., 0] + 1j * mat[..., 1]

    def execute(self, iterations=1):
        self.lib.ref_dgm_execute(self.h, iterations)

    def measure(self, qubit):
        return self.lib.ref_dgm_measure(self.h, qubit)

    def seed(self, s):
        self.lib.ref_seed_rng(s)

    def uniform_sample(self, s):
        """The sample measure() draws first after seed(s); leaves the generator seeded with s."""
        return self.lib.ref_uniform_sample(s)

    def colapse(self, qubit, value):
        self.lib.ref_dgm_colapse(self.h, qubit, value)

    def measure_many(self, qubits):
        """DGM::measure(vector<int>): {index & mask: probability}."""
        q = (C.c_int * len(qubits))(*qubits)
        cap = 1 << len(qubits)
        keys = (C.c_long * cap)()
        probs = (C.c_double * cap)()
        n = self.lib.ref_dgm_measure_many(self.h, q, len(qubits), keys, probs, cap)
        return {int(keys[k]): float(probs[k]) for k in range(min(n, cap))}
