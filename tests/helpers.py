"""Shared helpers: run a CircuitSpec on the engine and on the oracle."""
from __future__ import annotations

import math

import numpy as np

from oracle import circuit_lang as cl
from oracle import cpu

TOL_F64 = 1e-12      # max |amplitude error| vs the FP64 oracle
TOL_F32 = 2e-5       # max |amplitude error| vs the FP32 oracle (same op order, FP32 rounding)
REG_BITS = {"f64": 4, "f32": 5}   # amplitudes a thread keeps in registers = 2^R


def min_tiled_qubits(prec, warp_bits=0):
    """Smallest state that runs on the register-tile pass kernel with this many warp bits."""
    return 5 + REG_BITS[prec] + warp_bits


def oracle_state(spec, prec="f64", init=None):
    c = spec.build(cl.Circuit())
    n = spec.qubits
    s0 = cpu.basis_state(n, spec.init_index) if init is None else init
    return cpu.run_serial(s0, n, c.as_arrays(), prec=prec)


def engine_state(sq, spec, prec="f64", init=None, iterations=1, **plan_kw):
    c = spec.build(sq.Circuit())
    st = sq.State(spec.qubits, prec)
    if init is None:
        st.set_basis(spec.init_index)
    else:
        st.upload(init)
    plan = sq.Plan(c, spec.qubits, prec, **plan_kw)
    st.execute(plan, iterations)
    out = st.download()
    st.free()
    return out, plan.stats()


def random_state(n, seed, dtype=np.complex128):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    v /= np.linalg.norm(v)
    return v.astype(dtype)


def fidelity_gap(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    ov = np.vdot(a, b)
    return 1.0 - abs(ov) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def random_gate_circuit_spec(n, n_ops, seed, max_controls=3):
    """Random ops of every matrix class on every target, random controls."""
    from simulador_quantico_b200.workloads import CircuitSpec

    rng = np.random.default_rng(seed)
    gates = {}
    steps = []
    kinds = ["dense", "real", "diag", "phase", "anti", "swap"]
    for i in range(n_ops):
        kind = kinds[i % len(kinds)]
        a = rng.uniform(0, 2 * math.pi, 4)
        if kind == "dense":
            th = a[0]
            m = [np.cos(th) * np.exp(1j * a[1]), -np.sin(th) * np.exp(1j * a[2]),
                 np.sin(th) * np.exp(1j * (a[1] + a[3])), np.cos(th) * np.exp(1j * (a[2] + a[3]))]
        elif kind == "real":
            m = [np.cos(a[0]), -np.sin(a[0]), np.sin(a[0]), np.cos(a[0])]
        elif kind == "diag":
            m = [np.exp(1j * a[0]), 0, 0, np.exp(1j * a[1])]
        elif kind == "phase":
            m = [1, 0, 0, np.exp(1j * a[0])]
        elif kind == "anti":
            m = [0, np.exp(1j * a[0]), np.exp(1j * a[1]), 0]
        else:
            m = [0, 1, 1, 0]
        name = f"g{i}"
        gates[name] = m
        tq = int(rng.integers(n))
        others = [q for q in range(n) if q != tq]
        k = int(rng.integers(0, max_controls + 1))
        ctrl = rng.choice(others, size=min(k, len(others)), replace=False) if k else []
        tok = ["ID"] * n
        for c in ctrl:
            tok[int(c)] = "Control1(1)" if rng.integers(2) else "Control1(0)"
        tok[tq] = f"Target1({name})" if len(ctrl) else name
        steps.append(",".join(tok))
    return CircuitSpec("random_gates", n, 0, gates, [(steps, 1, True)], {"seed": seed})
