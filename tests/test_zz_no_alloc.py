"""hgm_norm_noalloc: the FP64 norm for callers that cannot allocate device memory.

Some callers of this library run inside a host framework that owns every
device allocation, or while another thread is capturing a CUDA graph, and
cannot call cudaMalloc.  hgm_norm_noalloc keeps its reduction scratch in a
file-scope device array instead.  This test calls it through the C-ABI and
checks it against hgm_norm (the allocating entry point) on two calls in a
row, within the FP64 tolerance the other tests use (1e-12, relative).  The
file is named to be collected last, and the test runs the same alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import TOL_F64, random_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("qubits,prec", [(18, "f64"), (21, "f32"), (3, "f64")])
def test_norm_noalloc_matches_norm(sq, qubits, prec):
    lib = sq._lib.lib
    host = random_state(qubits, seed=qubits) * 1.7
    st = sq.State(qubits, prec).upload(host)
    out = sq.State(1, "f64")  # 32 bytes of device memory the caller owns for the result
    ref = st.norm()
    for call in range(2):
        out.set_basis(1)  # overwrite the result slot so each call must write it
        rc = lib.hgm_norm_noalloc(C.c_void_p(lib.hgm_state_device_ptr(st.h)), qubits, st.precision,
                                  C.c_void_p(lib.hgm_state_device_ptr(out.h)), None)
        assert rc == 0, sq._lib.last_error()
        sq.synchronize()
        got = out.download()[0].real
        assert abs(got - ref) <= TOL_F64 * ref, (call, got, ref)
    st.free()
    out.free()


def test_norm_noalloc_rejects_oversize(sq):
    lib = sq._lib.lib
    dummy = C.c_void_p(8)
    rc = lib.hgm_norm_noalloc(dummy, 35, 0, dummy, None)
    assert rc == 4
    assert "1..34" in sq._lib.last_error()
