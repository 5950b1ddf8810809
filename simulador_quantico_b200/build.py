"""Builds the engine's shared libraries in-tree with nvcc for sm_100a.

    libhgm_b200.so          engine: circuits, planner, kernels, C-ABI
    libhgm_dropin_f32.so    reference GPU-backend symbols, complex float
    libhgm_dropin_f64.so    reference GPU-backend symbols, complex double

Output: simulador_quantico_b200/lib/.  Run ``python simulador_quantico_b200/build.py``
(the package itself imports only once the libraries exist) or call ``build()``; a library is rebuilt when any source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}", "-ccbin", "g++"]

ENGINE_SRCS = ["circuit.cpp", "planner.cpp", "engine.cpp", "kernels.cu", "batch.cu", "server.cpp", "hostcopy.cpp"]
# Extra nvcc flags (e.g. -DHGM_MAXREG_F32=128) and an alternative output
# folder, for building tuning variants side by side.
EXTRA_FLAGS = os.environ.get("HGM_NVCC_EXTRA", "").split()


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    return "nvcc"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build(verbose: bool = False, ptxas_verbose: bool = False, lib_dir: Path | None = None) -> None:
    LIB = Path(lib_dir) if lib_dir else globals()["LIB"]
    LIB.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    nvcc = _nvcc()
    objdir = LIB / "obj"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in ENGINE_SRCS:
        s = CSRC / src
        o = objdir / (src + ".o")
        if _stale(o, [s, *headers]):
            extra = ["-Xptxas", "-v"] if (ptxas_verbose and src.endswith(".cu")) else []
            _run([nvcc, *ARCH, *NVCC_FLAGS, *EXTRA_FLAGS, *extra, "-c", s, "-o", o], verbose)
        objs.append(o)
    engine = LIB / "libhgm_b200.so"
    if _stale(engine, objs):
        _run([nvcc, *ARCH, "-shared", "-o", engine, *objs, "-Xlinker", "-soname=libhgm_b200.so", "-lpthread"],
             verbose)
    for prec, define in (("f32", []), ("f64", ["-DHGM_DROPIN_F64"])):
        so = LIB / f"libhgm_dropin_{prec}.so"
        src = CSRC / "dropin.cpp"
        if _stale(so, [src, engine, *headers]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", *define, f"-I{INCLUDE}", f"-I{CSRC}", src,
                  "-o", so, f"-L{LIB}", "-lhgm_b200", "-Wl,-rpath,$ORIGIN"], verbose)


if __name__ == "__main__":
    out = os.environ.get("HGM_LIB_OUT")
    build(verbose=True, ptxas_verbose="-v" in sys.argv, lib_dir=Path(out) if out else None)
