"""The C-ABI libraries load and export every symbol their headers declare (CPU only).

include/hgm_b200.h   -> simulador_quantico_b200/lib/libhgm_b200.so
include/hgm_dropin.h -> simulador_quantico_b200/lib/libhgm_dropin_{f32,f64}.so
No compute call is made here (no GPU in this container).
"""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "simulador_quantico_b200" / "lib"


def declared(header):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
        name = m.group(1)
        if name in {"if", "sizeof", "defined"}:
            continue
        # keep only declarations at statement start: preceded by a type
        start = text.rfind("\n", 0, m.start())
        line = text[start + 1:m.start()]
        if line.strip().startswith("#") or not line.strip():
            continue
        names.add(name)
    return sorted(names)


@pytest.mark.parametrize("name", declared("hgm_b200.h"))
def test_engine_exports(name):
    lib = C.CDLL(str(LIB / "libhgm_b200.so"))
    assert hasattr(lib, name), name


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_dropin_exports(prec):
    lib = C.CDLL(str(LIB / f"libhgm_dropin_{prec}.so"))
    names = declared("hgm_dropin.h")
    assert set(names) == {"setDevice", "GpuExecutionWrapper", "ProjectState", "GetState"}
    for n in names:
        assert hasattr(lib, n), n


def test_package_import_needs_library():
    """The product path has no CPU fallback: the package imports only with its .so present."""
    import simulador_quantico_b200._lib as L

    assert L.ENGINE.exists()
    assert L.lib is not None


def test_plan_building_is_host_only():
    """Plans are built without touching the GPU (upload happens at first execute)."""
    import simulador_quantico_b200 as sq
    from simulador_quantico_b200 import workloads as wl

    spec = wl.random_layered(30, 2, seed=1)
    c = spec.build(sq.Circuit())
    p = sq.Plan(c, 30, "f64")
    s = p.stats()
    assert s["passes"] >= 3 and s["ops"] <= len(c)


@pytest.mark.parametrize("tuning,words", [((4, 8, 1, 32, 2), "2*block_size*repeat_count"),
                                          ((8, 6, 1, 16, 2), "gpu_region_bits (6)"),
                                          ((4, 8, 5, 64, 2), "gpu_count (5)")])
def test_dropin_tuning_rules_exit(tuning, words):
    """GpuExecutionWrapper refuses the tuning DGM::validateTuning refuses
    (src/core/dgm_core.cpp:199-240) with the same message start and exit
    status 1, before any device work (run in a child process, no GPU)."""
    import subprocess
    import sys

    code = f"""
import ctypes as C
L = C.CDLL({str(LIB / 'libhgm_dropin_f64.so')!r})
L.GpuExecutionWrapper.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 7
L.GpuExecutionWrapper.restype = C.c_void_p
buf = (C.c_double * 2)()
L.GpuExecutionWrapper(C.addressof(buf), None, 1, *{tuning!r}, 1)
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1, (r.returncode, r.stdout, r.stderr)
    assert "Erro de tuning" in r.stdout and words in r.stdout, r.stdout
