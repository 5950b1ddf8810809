"""Generates tests/golden/*.npz from the reference's own engine.

Run in a container that has the reference tree built into oracle/_ref
(``bash oracle/build_ref.sh``):

    python tests/golden/make_golden.py

Each fixture holds, for one circuit, the compiled PT list the reference's
parser produced (target bit, control mask/value, FP64 matrix) and the final
state of the reference's FP64-widened t_CPU backend
(DGM::CpuExecution1, src/core/dgm_cpu_exec.cpp:11-35) and of its unmodified
FP32 t_PAR_CPU backend (PCpuExecution1, src/core/dgm_par_exec.cpp:82-132).
The circuits are the reference's own test cases (tests/test_gates.cpp:43-90,
tests/smoke_test.sh:70-76) and small instances of the benchmark shapes.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import circuit_lang as cl  # noqa: E402
from oracle import cpu  # noqa: E402
from simulador_quantico_b200 import workloads as wl  # noqa: E402


def cases():
    out = []
    # tests/test_gates.cpp:43-90 -- one fixture per start state
    gate_cases = [("cnot", 2, cl.CNot(2, 0, 1, 1)), ("toffoli", 3, cl.Toffoli(3, 0, 1, 2, 3)),
                  ("controlledN", 4, cl.ControlledN(4, [0, 1, 2], 3, "X", -1)),
                  ("controlled1_ctrl0", 2, cl.Controlled1(2, 0, 1, "X", 0))]
    for name, n, step in gate_cases:
        for start in range(1 << n):
            out.append((f"gates_{name}_{start}", wl.CircuitSpec(name, n, start, {}, [([step], 1, True)])))
    # tests/smoke_test.sh:70-76 shapes
    for n in (10, 14):
        out.append((f"hadamard_{n}", wl.hadamard_benchmark(n, 3)))
    out.append(("grover_ref_9", wl.grover_reference(9, 42 % 256)))
    out.append(("grover_ref_11_4it", wl.grover_reference(11, 300, 4)))
    out.append(("layered_10", wl.random_layered(10, 3, seed=11)))
    out.append(("layered_13", wl.random_layered(13, 2, seed=12)))
    out.append(("qft_8", wl.qft(8, 77)))
    out.append(("grover_search_9", wl.grover_search(9, 300)))
    return out


def run_reference(spec, prec, exec_type, threads=4):
    r = cpu.RefDGM(spec.qubits, prec)
    r.tuning(exec_type, thread_count=threads)
    for name, m in spec.gates.items():
        r.add_gate(name, m)
    r.set_memory_value(spec.init_index)
    for steps, it, reset in spec.calls:
        r.set_function(steps, it, reset)
    pts = r.pts()
    r.execute(1)
    s = r.state()
    r.close()
    return pts, s


def main():
    if not cpu.ref_available("f64") or not cpu.ref_available("f32"):
        raise SystemExit("oracle/_ref is not built: run `bash oracle/build_ref.sh` first")
    for name, spec in cases():
        (t, cm, cv, m), s64 = run_reference(spec, "f64", cpu.RefDGM.T_CPU)
        _, s32 = run_reference(spec, "f32", cpu.RefDGM.T_PAR_CPU)
        np.savez_compressed(HERE / f"{name}.npz", qubits=spec.qubits, init_index=spec.init_index, target=t, cmask=cm,
                            cval=cv, matrix=m, state_f64=s64, state_f32_par=s32.astype(np.complex64))
    print(f"wrote {len(cases())} fixtures to {HERE}")


if __name__ == "__main__":
    main()
