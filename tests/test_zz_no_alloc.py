"""hgm_norm_noalloc: the FP64 norm for callers that cannot allocate device memory.

Some callers of this library run inside a host framework that owns every
device allocation and hands the library only its buffers, or run while
another thread is capturing a CUDA graph, where an allocation would break
the capture; they cannot call cudaMalloc.  hgm_norm_noalloc keeps its
reduction scratch in a file-scope device array instead and writes its result
to one device double the caller provides.

This test calls it through the C-ABI on two calls in a row and checks:
  * the result against the host norm of the uploaded array (np.vdot of the
    values as the device holds them, in FP64), within the FP64 tolerance the
    other tests use (1e-12, relative), and against hgm_norm, the allocating
    entry point, at the same tolerance;
  * that only the 8-byte result slot is written: a guard double right after
    it, and the rest of the caller's buffer, keep their values.
The file is named to be collected last, and the test runs the same alone in
a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import TOL_F64, random_state

pytestmark = pytest.mark.gpu

GUARD = 12345.678


@pytest.mark.parametrize("qubits,prec", [(18, "f64"), (21, "f32"), (3, "f64"), (27, "f32")])
def test_norm_noalloc_matches_host_norm(sq, qubits, prec):
    lib = sq._lib.lib
    dt = np.complex128 if prec == "f64" else np.complex64
    host = (random_state(qubits, seed=qubits) * 1.7).astype(dt)
    st = sq.State(qubits, prec).upload(host)
    held = host.astype(np.complex128)
    want = float(np.vdot(held, held).real)
    ref = st.norm()
    # the caller's buffer: result slot (8 bytes), then a guard double, then 16 more bytes
    buf = sq.State(1, "f64")
    fill = np.array([complex(-1.0, GUARD), complex(GUARD + 1, GUARD + 2)], dtype=np.complex128)
    for call in range(2):
        buf.upload(fill)  # every call must write the slot itself
        rc = lib.hgm_norm_noalloc(C.c_void_p(lib.hgm_state_device_ptr(st.h)), qubits, st.precision,
                                  C.c_void_p(lib.hgm_state_device_ptr(buf.h)), None)
        assert rc == 0, sq._lib.last_error()
        sq.synchronize()
        got = buf.download()
        assert abs(got[0].real - want) <= TOL_F64 * want, (call, got[0].real, want)
        assert abs(got[0].real - ref) <= TOL_F64 * ref, (call, got[0].real, ref)
        assert got[0].imag == GUARD, (call, got[0].imag)
        assert got[1] == fill[1], (call, got[1])
    st.free()
    buf.free()


def test_norm_noalloc_rejects_oversize(sq):
    lib = sq._lib.lib
    dummy = C.c_void_p(8)
    rc = lib.hgm_norm_noalloc(dummy, 35, 0, dummy, None)
    assert rc == 4
    assert "1..34" in sq._lib.last_error()
