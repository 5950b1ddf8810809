"""Python face of the engine: circuits, plans, device states and a DGM mirror.

Everything here calls libhgm_b200.so through ctypes (_lib.py); there is no
Python or CPU compute path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import HGM_F32, HGM_F64, PlanOpts, check, lib

PREC = {"f64": HGM_F64, "f32": HGM_F32, HGM_F64: HGM_F64, HGM_F32: HGM_F32}
NP_DTYPE = {HGM_F64: np.complex128, HGM_F32: np.complex64}

_initialised = False


def init(device: int = 0):
    """Creates the CUDA context on `device` (setDevice, src/core/kernel.cu:31-33)."""
    global _initialised
    if not _initialised:
        check(lib.hgm_init(device))
        _initialised = True


def _m8(m) -> "C.Array":
    m = np.asarray(m, dtype=np.complex128).reshape(4)
    buf = (C.c_double * 8)()
    for k in range(4):
        buf[2 * k] = float(m[k].real)
        buf[2 * k + 1] = float(m[k].imag)
    return buf


class Circuit:
    """Compiled op list built with the reference's circuit language.

    ``add_gate`` = Gates::addGate (src/core/gates.cpp:42-60),
    ``set_function`` = DGM::setFunction (src/core/dgm_parser.cpp:29-66).
    """

    def __init__(self):
        self.h = lib.hgm_circuit_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib.hgm_circuit_free(self.h)
            self.h = None

    def add_gate(self, name: str, m) -> bool:
        rc = lib.hgm_circuit_add_gate(self.h, name.encode(), _m8(m))
        if rc < 0:
            raise _lib.HgmError(-rc, _lib.last_error())
        return rc == 1

    def set_function(self, steps, iterations: int = 1, reset: bool = True):
        if not isinstance(steps, str):
            steps = ";".join(steps)
        check(lib.hgm_circuit_set_function(self.h, steps.encode(), iterations, 1 if reset else 0))
        return self

    def append_op(self, target, cmask, cval, m):
        check(lib.hgm_circuit_append_op(self.h, target, cmask, cval, _m8(m)))

    @property
    def qubits(self) -> int:
        return lib.hgm_circuit_qubits(self.h)

    def __len__(self):
        return lib.hgm_circuit_num_ops(self.h)

    def ops(self):
        n = len(self)
        t = np.empty(n, np.int32)
        cm = np.empty(n, np.int64)
        cv = np.empty(n, np.int64)
        m = np.empty(8 * n, np.float64)
        if n:
            check(lib.hgm_circuit_get_ops(self.h, t.ctypes.data_as(C.POINTER(C.c_int32)),
                                          cm.ctypes.data_as(C.POINTER(C.c_int64)),
                                          cv.ctypes.data_as(C.POINTER(C.c_int64)),
                                          m.ctypes.data_as(C.POINTER(C.c_double))))
        mm = m.reshape(n, 4, 2)
        return t, cm, cv, mm[..., 0] + 1j * mm[..., 1]

    def ref_pts(self, precision="f64"):
        """NULL-terminated PT** in the reference's struct layout.  The arrays
        belong to this circuit: the pointer is valid while the circuit lives."""
        p = lib.hgm_circuit_ref_pts(self.h, PREC[precision])
        if not p:
            raise _lib.HgmError(1, _lib.last_error())
        return p


def plan_opts(precision="f64", **kw) -> PlanOpts:
    o = PlanOpts()
    lib.hgm_plan_default_opts(C.byref(o), PREC[precision])
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Plan:
    def __init__(self, circuit: Circuit, qubits: int, precision="f64", **kw):
        self.h = C.c_void_p()
        self.precision = PREC[precision]
        self.qubits = qubits
        self.opts = plan_opts(precision, **kw)
        check(lib.hgm_plan_create(circuit.h, qubits, C.byref(self.opts), C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            lib.hgm_plan_free(self.h)
            self.h = None

    def upload(self):
        """Copy the plan's device records now rather than at first use."""
        check(lib.hgm_plan_upload(self.h))
        return self

    def status(self):
        """Waits for the device; raises if the plan's last chained execution gave up a bounded wait."""
        check(lib.hgm_plan_status(self.h))
        return self

    def stats(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        check(lib.hgm_plan_stats(self.h, *[C.byref(x) for x in v]))
        wb, small = C.c_int(), C.c_int()
        nph, nb, npa = C.c_int64(), C.c_int64(), C.c_int64()
        passes = C.c_void_p()
        check(lib.hgm_plan_export(self.h, C.byref(passes), C.byref(npa), None, C.byref(nph), None, C.byref(nb),
                                  C.byref(wb), C.byref(small)))
        # bytes copied to the device when the plan is created: op records and phase table
        upload = nb.value + 16 * nph.value
        # register bits from the first pass's tile bits (struct PassArgs: n, k, ...): k = 5 + R + W
        reg_bits = 4 if self.precision == HGM_F64 else 5
        if npa.value and passes.value:
            reg_bits = C.cast(passes, C.POINTER(C.c_int32))[1] - 5 - wb.value
        return dict(ops=v[0].value, passes=v[1].value, phases=v[2].value, transposes=v[3].value,
                    warp_bits=wb.value, reg_bits=reg_bits, small=bool(small.value), upload_bytes=upload)


class State:
    """A device-resident state vector."""

    def __init__(self, qubits: int, precision="f64"):
        init()
        self.qubits = qubits
        self.precision = PREC[precision]
        self.h = C.c_void_p()
        self.owner = None
        check(lib.hgm_state_create(qubits, self.precision, C.byref(self.h)))

    @classmethod
    def view(cls, handle, qubits, precision, owner):
        """A non-owning handle on a state another object (batch, server) owns."""
        st = cls.__new__(cls)
        st.qubits, st.precision, st.h, st.owner = qubits, PREC[precision], C.c_void_p(handle), owner
        return st

    def free(self):
        if getattr(self, "h", None):
            if self.owner is None:
                lib.hgm_state_free(self.h)
            self.h = None

    def __del__(self):
        self.free()

    @property
    def nbytes(self):
        return (1 << self.qubits) * (16 if self.precision == HGM_F64 else 8)

    def set_basis(self, index: int):
        check(lib.hgm_state_set_basis(self.h, index))
        return self

    def upload(self, host):
        arr = np.ascontiguousarray(np.asarray(host, dtype=NP_DTYPE[self.precision]))
        check(lib.hgm_state_upload(self.h, arr.ctypes.data, arr.nbytes))
        return self

    def download(self, out=None):
        if out is None:
            out = np.empty(1 << self.qubits, dtype=NP_DTYPE[self.precision])
        check(lib.hgm_state_download(self.h, out.ctypes.data, out.nbytes))
        return out

    def execute(self, plan: Plan, iterations: int = 1, stream=None):
        check(lib.hgm_execute(self.h, plan.h, iterations, stream))
        return self

    def norm(self) -> float:
        v = C.c_double()
        check(lib.hgm_norm(self.h, C.byref(v)))
        return v.value

    def prob_one(self, bit: int) -> float:
        v = C.c_double()
        check(lib.hgm_prob_one(self.h, bit, C.byref(v)))
        return v.value

    def measure_qubit(self, qubit: int, sample: float):
        o, p = C.c_int(), C.c_double()
        check(lib.hgm_measure_qubit(self.h, qubit, sample, C.byref(o), C.byref(p)))
        return o.value, p.value

    def collapse_qubit(self, qubit: int, value: int) -> float:
        p = C.c_double()
        check(lib.hgm_collapse_qubit(self.h, qubit, value, C.byref(p)))
        return p.value

    def marginal_probs(self, mask: int):
        """Probabilities of every value of the mask bits (bit j of the index = j-th lowest mask bit)."""
        out = np.empty(1 << bin(mask).count("1"), dtype=np.float64)
        check(lib.hgm_marginal_probs(self.h, mask, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    def marginal_argmax(self, mask: int):
        a, p = C.c_int64(), C.c_double()
        check(lib.hgm_marginal_argmax(self.h, mask, C.byref(a), C.byref(p)))
        return a.value, p.value

    def inner(self, other: "State"):
        re, im = C.c_double(), C.c_double()
        check(lib.hgm_inner(self.h, other.h, C.byref(re), C.byref(im)))
        return complex(re.value, im.value)

    def max_abs_diff(self, other: "State") -> float:
        v = C.c_double()
        check(lib.hgm_max_abs_diff(self.h, other.h, C.byref(v)))
        return v.value

    def scale(self, f: float):
        check(lib.hgm_scale(self.h, f))


class Batch:
    """Many circuits in one persistent kernel replayed from a CUDA graph (include/hgm_b200.h)."""

    def __init__(self, precision="f32", warp_bits=-1):
        init()
        self.precision = PREC[precision]
        self.h = C.c_void_p()
        self.qubits = []
        check(lib.hgm_batch_create(self.precision, warp_bits, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            lib.hgm_batch_free(self.h)
            self.h = None

    def add(self, circuit: Circuit, qubits: int, init_index: int = 0) -> int:
        j = C.c_int()
        check(lib.hgm_batch_add(self.h, circuit.h, qubits, init_index, C.byref(j)))
        self.qubits.append(qubits)
        return j.value

    def finalize(self):
        check(lib.hgm_batch_finalize(self.h))
        return self

    def run(self, stream=None):
        check(lib.hgm_batch_run(self.h, stream))
        return self

    def autotune(self, stream=None) -> dict:
        """Picks the tile size and resident low bits by timing graph replays."""
        w, lo, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib.hgm_batch_autotune(self.h, stream, C.byref(w), C.byref(lo), C.byref(ms)))
        return dict(warp_bits=w.value, low_bits=lo.value, ms=ms.value)

    def set_inputs(self, init_index, stream=None):
        """Every job's initial basis index for the next runs (int64 array, one per job)."""
        a = np.ascontiguousarray(init_index, dtype=np.int64)
        check(lib.hgm_batch_set_inputs(self.h, a.ctypes.data_as(C.POINTER(C.c_int64)), stream))
        self._inputs = a  # the copy is asynchronous: keep the buffer alive
        return self

    def download(self, host: "PinnedArray", stream=None):
        """Every job's state, back to back in job order, into `host` (asynchronous)."""
        check(lib.hgm_batch_download(self.h, C.c_void_p(host.ptr), host.nbytes, stream))
        return self

    def check(self):
        check(lib.hgm_batch_check(self.h))

    def inject_stall(self, task: int, wait_ns: int = 0):
        """Test hook: task `task` waits on a completion that never comes, every wait limited to wait_ns;
        task < 0 restores the normal table (hgm_batch_inject_stall)."""
        check(lib.hgm_batch_inject_stall(self.h, task, wait_ns))
        return self

    def size(self) -> dict:
        j, t, it, ab, pb = C.c_int(), C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.hgm_batch_size(self.h, C.byref(j), C.byref(t), C.byref(it), C.byref(ab), C.byref(pb)))
        return dict(jobs=j.value, tasks=t.value, items=it.value, arena_bytes=ab.value, pass_bytes=pb.value)

    def state(self, job: int) -> State:
        h = lib.hgm_batch_state(self.h, job)
        if not h:
            raise _lib.HgmError(1, _lib.last_error())
        return State.view(h, self.qubits[job], self.precision, owner=self)


class Server:
    """Continuous-batching server (include/hgm_b200.h, serving mode)."""

    def __init__(self, precision="f32", budget_bytes=150 << 30, max_inflight=32, keep_states=False, warp_bits=-1,
                 order="arrival"):
        init()
        o = _lib.ServerOpts()
        lib.hgm_server_default_opts(C.byref(o), PREC[precision])
        o.budget_bytes, o.max_inflight, o.keep_states, o.warp_bits = budget_bytes, max_inflight, int(keep_states), warp_bits
        o.order = {"arrival": _lib.HGM_ORDER_ARRIVAL, "work_first": _lib.HGM_ORDER_WORK_FIRST}[order]
        self.precision = PREC[precision]
        self.h = C.c_void_p()
        self.qubits = {}
        check(lib.hgm_server_create(C.byref(o), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            lib.hgm_server_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, circuit: Circuit, qubits: int, init_index: int = 0, result_mask: int = 0) -> int:
        rid = C.c_int64()
        check(lib.hgm_server_submit(self.h, circuit.h, qubits, init_index, result_mask, C.byref(rid)))
        self.qubits[rid.value] = qubits
        return rid.value

    def submit_plan(self, plan: "Plan", init_index: int = 0, result_mask: int = 0) -> int:
        """Queues an already built (device-resident) plan, which must not run
        elsewhere until this request's result is polled.  The request leases
        the plan: freeing it (or letting it be collected) before then only
        marks it, and the server frees it when the request is done."""
        rid = C.c_int64()
        check(lib.hgm_server_submit_plan(self.h, plan.h, init_index, result_mask, C.byref(rid)))
        self.qubits[rid.value] = plan.qubits
        return rid.value

    def poll(self, max_results=256, wait_ms=0):
        buf = (_lib.Result * max_results)()
        n = C.c_int()
        check(lib.hgm_server_poll(self.h, buf, max_results, C.byref(n), wait_ms))
        return [dict(id=r.id, status=r.status, qubits=r.qubits, latency_s=r.latency_s, queue_s=r.queue_s,
                     exec_s=r.exec_s, norm=r.norm, argmax=r.argmax, pmax=r.pmax) for r in buf[:n.value]]

    def pending(self):
        q, f, b = C.c_int(), C.c_int(), C.c_int64()
        check(lib.hgm_server_pending(self.h, C.byref(q), C.byref(f), C.byref(b)))
        return dict(queued=q.value, inflight=f.value, bytes_in_use=b.value)

    def drain(self, expected, timeout_s=600.0):
        """Collects results until `expected` have arrived."""
        import time as _t

        out, t0 = [], _t.time()
        while len(out) < expected:
            out += self.poll(wait_ms=50)
            if _t.time() - t0 > timeout_s:
                raise TimeoutError(f"{len(out)}/{expected} results after {timeout_s} s")
        return out

    def result_state(self, rid: int) -> State:
        h = lib.hgm_server_result_state(self.h, rid)
        if not h:
            raise _lib.HgmError(1, _lib.last_error())
        return State.view(h, self.qubits[rid], self.precision, owner=self)

    def release(self, rid: int):
        check(lib.hgm_server_release(self.h, rid))


def synchronize():
    check(lib.hgm_synchronize())


def mem_info():
    """(free, total) device memory in bytes."""
    init()
    f, t = C.c_int64(), C.c_int64()
    check(lib.hgm_mem_info(C.byref(f), C.byref(t)))
    return f.value, t.value


def kernel_launches() -> int:
    return lib.hgm_kernel_launches()


class Timer:
    """CUDA events around the work queued on the library stream."""

    def __enter__(self):
        check(lib.hgm_timer_start())
        return self

    def __exit__(self, *a):
        ms = C.c_double()
        check(lib.hgm_timer_stop(C.byref(ms)))
        self.ms = ms.value


# ---------------------------------------------------------------------------
# DGM mirror (include/core/dgm.h:65-163) with a device-resident state
# ---------------------------------------------------------------------------

T_CPU, T_PAR_CPU, T_GPU, T_HYBRID = 0, 1, 2, 3


@dataclass
class DGM:
    """The reference's DGM facade on the B200 engine.

    Same fields and call sequence as include/core/dgm.h:65-163 (qubits,
    exec_type, tuning fields, allocateMemory, setMemoryValue, setFunction,
    execute, measure), with the state kept on the device.  Only exec_type
    t_GPU is provided; the tuning fields are validated like
    DGM::validateTuning (src/core/dgm_core.cpp:177-241).
    """

    qubits: int = 0
    exec_type: int = T_GPU
    precision: str = "f64"
    gpu_count: int = 1
    gpu_region_bits: int = 8
    gpu_coalesced_bits: int = 4
    block_size: int = 64
    repeat_count: int = 2
    circuit: Circuit = field(default_factory=Circuit)
    state: State | None = None

    def allocateMemory(self):
        self.state = State(self.qubits, self.precision)
        self.state.set_basis(0)

    def setMemoryValue(self, pos: int):
        self.state.set_basis(pos)

    def setFunction(self, steps, iterations=1, reset=True):
        self.circuit.set_function(steps, iterations, reset)

    def validateTuning(self):
        if self.exec_type != T_GPU:
            raise ValueError(f"exec_type {self.exec_type} is not provided by the B200 engine (t_GPU only)")
        self.gpu_region_bits = min(self.gpu_region_bits, self.qubits)
        if 2 * self.block_size * self.repeat_count != (1 << self.gpu_region_bits):
            raise ValueError("2*block_size*repeat_count must equal 2^gpu_region_bits")
        if self.gpu_region_bits < self.gpu_coalesced_bits:
            raise ValueError("gpu_region_bits must be >= gpu_coalesced_bits")

    def execute(self, iterations=1):
        self.validateTuning()
        plan = Plan(self.circuit, self.qubits, self.precision)
        self.state.execute(plan, iterations)
        return self.state

    def executeFunction(self, steps, iterations=1):
        self.setFunction(steps)
        return self.execute(iterations)

    def measure(self, qubit_pos: int, sample: float) -> int:
        """DGM::measure(int) with the uniform sample supplied by the caller."""
        outcome, _ = self.state.measure_qubit(qubit_pos, sample)
        return outcome

    def colapse(self, qubit_pos: int, value: int) -> float:
        """DGM::colapse (src/core/dgm_core.cpp:129-146); returns the probability collapsed onto."""
        return self.state.collapse_qubit(qubit_pos, value)

    def measure_positions(self, qubit_positions) -> dict:
        """DGM::measure(vector<int>) (src/core/dgm_core.cpp:150-162): {index & mask: probability}."""
        bits = sorted(self.qubits - 1 - q for q in qubit_positions)
        mask = 0
        for b in bits:
            mask |= 1 << b
        probs = self.state.marginal_probs(mask)
        out = {}
        for x, p in enumerate(probs):
            key = 0
            for j, b in enumerate(bits):
                key |= ((x >> j) & 1) << b
            out[key] = float(p)
        return out

    def host_state(self):
        return self.state.download()


class PinnedArray:
    """A numpy array in page-locked host memory (hgm_pinned_alloc)."""

    def __init__(self, shape, dtype):
        init()
        dt = np.dtype(dtype)
        n = int(np.prod(shape)) * dt.itemsize
        p = C.c_void_p()
        check(lib.hgm_pinned_alloc(max(n, 1), C.byref(p)))
        self.ptr, self.nbytes = p.value, n
        buf = (C.c_char * max(n, 1)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)

    def __del__(self):
        if getattr(self, "ptr", None):
            self.array = None
            lib.hgm_pinned_free(C.c_void_p(self.ptr))
            self.ptr = None
