"""Python restatement of the reference's circuit language (test oracle only).

TEST INFRASTRUCTURE: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg, to check results against; the product never
imports it.

Restates, function by function, how the reference turns gate strings into
the NULL-terminated PT list that every backend consumes:

* ``tokenize``            Tokenize, src/core/dgm_parser.cpp:10-26
* ``Gates``               Gates::init/addGate/getMatrix, src/core/gates.cpp:23-60
* ``gen_groups``          DGM::genGroups, src/core/dgm_parser.cpp:70-114
* ``gen_pts``             DGM::genPTs, src/core/dgm_parser.cpp:118-169
* ``Circuit.set_function``DGM::setFunction, src/core/dgm_parser.cpp:29-66
                          (per-step sort with the comparators of
                          src/core/common.cpp:166-178)
* step generators         CNot/Toffoli/Controlled1/Controlled2/ControlledN/
                          Pauli_X/Pauli_Z/Hadamard/concatena,
                          src/core/gates.cpp:69-163
* algorithm builders      HadamardNQubits (src/algorithms/lib_general.cpp:15-47),
                          Grover/Oracle1/ControledZ
                          (src/algorithms/lib_grover.cpp:15-91)

A compiled op is a tuple ``(target_bit, control_mask, control_value, m)``
with ``m`` a numpy complex128 array ``[m00, m01, m10, m11]`` (row-major).
Index bit ``b`` of the state belongs to circuit qubit ``n-1-b``.
"""
from __future__ import annotations

import cmath
import math
from dataclasses import dataclass, field

import numpy as np


def tokenize(text: str, delimiters: str = ",") -> list[str]:
    """Split on any delimiter character, skipping empty tokens (dgm_parser.cpp:10-26)."""
    out, cur = [], []
    for ch in text:
        if ch in delimiters:
            if cur:
                out.append("".join(cur))
                cur = []
        else:
            cur.append(ch)
    if cur:
        out.append("".join(cur))
    return out


def _strtol_prefix(s: str) -> int:
    """C strtol(s, &end, 10) on a prefix: optional sign then digits, else 0."""
    s = s.lstrip()
    i, sign = 0, 1
    if i < len(s) and s[i] in "+-":
        sign = -1 if s[i] == "-" else 1
        i += 1
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    return sign * int(s[i:j]) if j > i else 0


class Gates:
    """Named 2x2 matrices (gates.cpp:23-60); FP64 values.

    R_k = diag(1, e^{i*pi/2^(k-1)}) as the reference's cpowf(M_E, M_PI*I/2^(k-1)).
    ``add_gate`` never overwrites an existing name (gates.cpp:49-50).
    """

    def __init__(self):
        self.table: dict[str, np.ndarray] = {}
        s = 1.0 / math.sqrt(2.0)
        self.add_gate("H", s, s, s, -s)
        self.add_gate("X", 0.0, 1.0, 1.0, 0.0)
        self.add_gate("Z", 1.0, 0.0, 0.0, -1.0)
        self.add_gate("Y", 0.0, 1j, -1j, 0.0)
        self.add_gate("R1", 1.0, 0.0, 0.0, cmath.exp(1j * math.pi))
        self.add_gate("R2", 1.0, 0.0, 0.0, cmath.exp(1j * math.pi / 2.0))
        self.add_gate("R3", 1.0, 0.0, 0.0, cmath.exp(1j * math.pi / 4.0))

    def add_gate(self, name, a0, a1, a2, a3) -> bool:
        if name in self.table:
            return False
        self.table[name] = np.array([a0, a1, a2, a3], dtype=np.complex128)
        return True

    def get(self, name: str):
        return self.table.get(name)


@dataclass
class Group:
    ops: list = field(default_factory=list)
    pos_ops: list = field(default_factory=list)
    ctrl: list = field(default_factory=list)
    pos_ctrl: list = field(default_factory=list)


def gen_groups(step: str):
    """DGM::genGroups (dgm_parser.cpp:70-114): returns (groups, qubits)."""
    ops = tokenize(step, ",")
    qubits = len(ops)
    groups: dict[int, Group] = {}
    for qubit_pos, token in enumerate(ops):
        c = token.find("Control")
        t = token.find("Target")
        paren = token.find("(") + 1
        if c != -1:
            num = _strtol_prefix(token[7:])
            val = _strtol_prefix(token[paren:])
            g = groups.setdefault(num, Group())
            g.ctrl.append(val)
            g.pos_ctrl.append(qubit_pos)
        elif t != -1:
            num = _strtol_prefix(token[6:])
            name = token[paren:len(token) - 1]
            g = groups.setdefault(num, Group())
            g.ops.append(name)
            g.pos_ops.append(qubit_pos)
        elif token != "ID":
            g = groups.setdefault(0, Group())
            g.ops.append(token)
            g.pos_ops.append(qubit_pos)
    return groups, qubits


def gen_pts(groups, qubits: int, gates: Gates):
    """DGM::genPTs (dgm_parser.cpp:118-169): one op per target, groups in key order.

    Returns a list of (span_start_bit, target_bit, cmask, cval, matrix).
    """
    out = []
    for key in sorted(groups):
        g = groups[key]
        cmask = cval = 0
        for val, pos in zip(g.ctrl, g.pos_ctrl):
            bit = qubits - pos - 1
            cmask += 1 << bit
            if val:
                cval += 1 << bit
        for name, pos in zip(g.ops, g.pos_ops):
            span = qubits - pos
            m = gates.get(name)
            if m is None:
                raise KeyError(f"unknown gate {name!r}")
            out.append((span, span - 1, cmask, cval, m))
    return out


class Circuit:
    """The PT list a DGM holds: set_function mirrors DGM::setFunction."""

    def __init__(self, gates: Gates | None = None):
        self.gates = gates or Gates()
        self.ops: list[tuple] = []
        self.qubits = 0

    def add_gate(self, name, m) -> bool:
        m = np.asarray(m, dtype=np.complex128).reshape(4)
        return self.gates.add_gate(name, *m)

    def set_function(self, steps, iterations: int = 1, reset: bool = True):
        if isinstance(steps, str):
            steps = tokenize(steps, ";")
        if reset:
            self.ops = []
        for _ in range(iterations):
            for idx, step in enumerate(steps):
                groups, self.qubits = gen_groups(step)
                pts = gen_pts(groups, self.qubits, self.gates)
                # odd steps: `increasing` (descending span_start_bit);
                # even steps: `decreasing` (ascending) -- common.cpp:166-178.
                pts.sort(key=lambda p: p[0], reverse=bool(idx % 2))
                self.ops.extend((p[1], p[2], p[3], p[4]) for p in pts)
        return self

    def as_arrays(self):
        n = len(self.ops)
        target = np.array([o[0] for o in self.ops], dtype=np.int32)
        cmask = np.array([o[1] for o in self.ops], dtype=np.int64)
        cval = np.array([o[2] for o in self.ops], dtype=np.int64)
        mat = np.zeros((n, 4), dtype=np.complex128)
        for i, o in enumerate(self.ops):
            mat[i] = o[3]
        return target, cmask, cval, mat


# ---- step generators (gates.cpp:69-163) --------------------------------

def concatena(step_ops, qubits, reverse=False):
    seq = step_ops[:qubits] if not reverse else list(reversed(step_ops[:qubits]))
    return ",".join(seq)


def CNot(qubits, ctrl, target, control_value=1):
    s = ["ID"] * qubits
    s[ctrl] = "Control1(1)" if control_value else "Control1(0)"
    s[target] = "Target1(X)"
    return concatena(s, qubits)


def Toffoli(qubits, c1, c2, target, control_value=3):
    s = ["ID"] * qubits
    s[c1] = "Control1(1)" if control_value >> 1 else "Control1(0)"
    s[c2] = "Control1(1)" if control_value & 1 else "Control1(0)"
    s[target] = "Target1(X)"
    return concatena(s, qubits)


def Controlled1(qubits, ctrl, target, op, control_value=1):
    s = ["ID"] * qubits
    s[ctrl] = "Control1(1)" if control_value else "Control1(0)"
    s[target] = f"Target1({op})"
    return concatena(s, qubits)


def Controlled2(qubits, c1, c2, target, op, control_value=3):
    s = ["ID"] * qubits
    s[c1] = "Control1(1)" if control_value & 2 else "Control1(0)"
    s[c2] = "Control1(1)" if control_value & 1 else "Control1(0)"
    s[target] = f"Target1({op})"
    return concatena(s, qubits)


def ControlledN(qubits, ctrls, target, op, control_value=-1):
    if control_value == -1:
        control_value = 2 ** len(ctrls) - 1
    s = ["ID"] * qubits
    for c in reversed(ctrls):
        s[c] = "Control1(1)" if control_value & 1 else "Control1(0)"
        control_value >>= 1
    s[target] = f"Target1({op})"
    return concatena(s, qubits)


def _fill(qubits, reg, width, name):
    s = ["ID"] * qubits
    for q in range(width):
        s[q + reg] = name
    return concatena(s, qubits)


def Pauli_X(qubits, reg, width=1):
    return _fill(qubits, reg, width, "X")


def Pauli_Z(qubits, reg, width=1):
    return _fill(qubits, reg, width, "Z")


def Hadamard(qubits, reg, width=1):
    return _fill(qubits, reg, width, "H")


# ---- algorithm builders -------------------------------------------------

def hadamard_benchmark(qubits: int, iterations: int = 3) -> Circuit:
    """HadamardNQubits (lib_general.cpp:33-34): H on every qubit, unrolled."""
    return Circuit().set_function(Hadamard(qubits, 0, qubits), iterations)


def Oracle1(qubits, search_value):
    """lib_grover.cpp:68-82: X on qubit 0 controlled on the search register."""
    s = [""] * qubits
    for q in range(qubits - 1, 0, -1):
        s[q] = "Control1(1)" if search_value & 1 else "Control1(0)"
        search_value >>= 1
    s[0] = "Target1(X)"
    return concatena(s, qubits)


def ControledZ(qubits):
    """lib_grover.cpp:84-91."""
    s = ["ID"] + ["Control1(1)"] * (qubits - 2) + ["Target1(Z)"]
    return concatena(s, qubits)


def grover_steps(qubits, search_value):
    """One Grover iteration as the list of steps lib_grover.cpp:37-51 builds."""
    steps = [Oracle1(qubits, search_value)]
    for q in range(1, qubits):
        steps.append(Hadamard(qubits, q, 1))
        steps.append(Pauli_X(qubits, q, 1))
    steps.append(ControledZ(qubits))
    for q in range(qubits - 1, 0, -1):
        steps.append(Pauli_X(qubits, q, 1))
        steps.append(Hadamard(qubits, q, 1))
    return steps


def grover_iterations(qubits):
    """(int)(M_PI/4*sqrt(1<<(qubits-1))), lib_grover.cpp:53."""
    return int(math.pi / 4.0 * math.sqrt(1 << (qubits - 1)))


def grover_circuit(qubits, search_value, iterations=None) -> Circuit:
    """Grover() (lib_grover.cpp:15-66): H on all, then the unrolled iterations.

    The initial state is |1 0...0> (setMemoryValue(1<<(qubits-1)), :31).
    """
    if iterations is None:
        iterations = grover_iterations(qubits)
    c = Circuit().set_function(Hadamard(qubits, 0, qubits))
    c.set_function(grover_steps(qubits, search_value), iterations, reset=False)
    return c
