"""The product's C++ circuit parser (libhgm_b200.so, no GPU needed) vs the reference.

Its compiled op lists must equal the reference parser's PT lists in the
golden fixtures (target bit, control mask/value exactly; matrices within
1e-15), and it must keep the reference's rules: Gates::addGate never
overwrites (src/core/gates.cpp:49-50), setFunction(reset=false) appends
(dgm_parser.cpp:43-44), steps alternate ascending/descending target order
(common.cpp:166-178), and the last step's width sets the qubit count
(dgm_parser.cpp:73).
"""
from pathlib import Path

import numpy as np
import pytest

import simulador_quantico_b200 as sq
from oracle import circuit_lang as cl
from simulador_quantico_b200 import workloads as wl
from tests.test_oracle import GOLDEN, golden_specs


@pytest.fixture(scope="module")
def specs():
    return golden_specs()


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_parser_matches_reference_pts(path, specs):
    g = np.load(path)
    c = specs[path.stem].build(sq.Circuit())
    t, cm, cv, m = c.ops()
    assert np.array_equal(t, g["target"])
    assert np.array_equal(cm, g["cmask"])
    assert np.array_equal(cv, g["cval"])
    assert np.abs(m - g["matrix"]).max(initial=0.0) < 1e-15


@pytest.mark.parametrize("builder", [lambda: wl.random_layered(17, 4, 3), lambda: wl.qft(11, 9),
                                     lambda: wl.grover_reference(10, 77, 3), lambda: wl.grover_search(10, 5, 2)])
def test_parser_matches_oracle_parser(builder):
    spec = builder()
    a = spec.build(sq.Circuit()).ops()
    b = spec.build(cl.Circuit()).as_arrays()
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert np.abs(a[3] - b[3]).max() < 1e-15


def test_add_gate_never_overwrites():
    c = sq.Circuit()
    assert c.add_gate("H", [1, 0, 0, 1]) is False
    assert c.add_gate("MyGate", [0, 1, 1, 0]) is True
    assert c.add_gate("MyGate", [1, 0, 0, 1]) is False
    c.set_function("MyGate,ID")
    t, cm, cv, m = c.ops()
    assert np.array_equal(m[0], [0, 1, 1, 0])


def test_reset_false_appends_and_width():
    c = sq.Circuit()
    c.set_function("H,H,H")
    c.set_function("X,ID,ID;ID,ID,Z", iterations=2, reset=False)
    t, _, _, _ = c.ops()
    # step 0 ascending (3 H: bits 0,1,2), then 2 x (X on bit 2, Z on bit 0)
    assert list(t) == [0, 1, 2, 2, 0, 2, 0]
    assert c.qubits == 3


def test_odd_steps_descending():
    c = sq.Circuit()
    c.set_function("H,ID,H,H;H,H,ID,H")
    t, _, _, _ = c.ops()
    assert list(t) == [0, 1, 3, 3, 2, 0]


def test_grouped_controls():
    c = sq.Circuit()
    c.set_function("Control1(1),Target2(X),Control2(0),Target1(H),ID")
    t, cm, cv, _ = c.ops()
    # group 1: control qubit 0 (bit 4) = 1, target qubit 3 (bit 1)
    # group 2: control qubit 2 (bit 2) = 0, target qubit 1 (bit 3)
    assert list(t) == [1, 3]
    assert list(cm) == [16, 4] and list(cv) == [16, 0]


def test_unknown_gate_is_an_error():
    c = sq.Circuit()
    with pytest.raises(sq.HgmError):
        c.set_function("NOPE,ID")


def test_ref_pts_layout():
    """hgm_circuit_ref_pts emits the reference's struct PT (include/core/common.h:57-90)."""
    import ctypes as C

    c = sq.Circuit()
    c.set_function("Control1(1),ID,Target1(X)")
    pp = C.cast(c.ref_pts("f64"), C.POINTER(C.c_void_p))
    assert pp[1] is None
    raw = C.string_at(pp[0], 80)
    target = int.from_bytes(raw[24:28], "little")
    cval = int.from_bytes(raw[32:40], "little")
    cmask = int.from_bytes(raw[40:48], "little")
    assert (target, cmask, cval) == (0, 4, 4)
    mat = C.cast(C.c_void_p(int.from_bytes(raw[8:16], "little")), C.POINTER(C.c_double))
    assert [mat[k] for k in range(8)] == [0, 0, 1, 0, 1, 0, 0, 0]
