"""Circuit builders for the benchmark workloads, in the reference's circuit language.

Each builder returns a ``CircuitSpec``: the gates to register, the
``setFunction`` calls to make and the initial basis index -- the same
sequence the reference's algorithm libraries perform on a DGM, so one spec
drives both this engine and any other consumer of the language.

* ``hadamard_benchmark``  HadamardNQubits (src/algorithms/lib_general.cpp:15-47)
* ``grover_reference``    Grover (src/algorithms/lib_grover.cpp:15-91), ancilla
                          on qubit 0
* ``grover_search``       ancilla-free Grover on m qubits: phase oracle on |w>,
                          diffusion H (I - 2|0><0|) H
* ``random_layered``      per layer Rz(theta) and Ry(phi) on every qubit, angles
                          uniform in [0, 2 pi) from the seed, then CNOT on a
                          random perfect matching
* ``qft``                 textbook QFT (H + controlled R_k, angle 2 pi / 2^k,
                          on all pairs, then qubit-reversal swaps as 3 CNOTs)
Matrices are computed in FP64.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class CircuitSpec:
    name: str
    qubits: int
    init_index: int = 0
    gates: dict = field(default_factory=dict)      # name -> [m00, m01, m10, m11]
    calls: list = field(default_factory=list)      # (steps: list[str], iterations, reset)
    meta: dict = field(default_factory=dict)

    def build(self, circuit):
        """Replays the spec on any object with add_gate(name, m) / set_function(steps, it, reset)."""
        for name, m in self.gates.items():
            circuit.add_gate(name, np.asarray(m, dtype=np.complex128))
        for steps, it, reset in self.calls:
            circuit.set_function(steps, it, reset)
        return circuit

    def n_ops_estimate(self):
        return sum(len(s) * it for s, it, _ in self.calls)


def _row(n, fill="ID"):
    return [fill] * n


def _join(tokens):
    return ",".join(tokens)


def hadamard_step(n, reg=0, width=None):
    width = n if width is None else width
    t = _row(n)
    for q in range(reg, reg + width):
        t[q] = "H"
    return _join(t)


def hadamard_benchmark(n: int, iterations: int = 3) -> CircuitSpec:
    """general.out: |0...0>, one step of H on every qubit unrolled `iterations` times."""
    return CircuitSpec("hadamard", n, 0, {}, [([hadamard_step(n)], iterations, True)])


def _single(n, q, name):
    t = _row(n)
    t[q] = name
    return _join(t)


def grover_oracle_step(n, search_value):
    """lib_grover.cpp:68-82."""
    t = [""] * n
    v = search_value
    for q in range(n - 1, 0, -1):
        t[q] = "Control1(1)" if v & 1 else "Control1(0)"
        v >>= 1
    t[0] = "Target1(X)"
    return _join(t)


def grover_controlled_z_step(n):
    """lib_grover.cpp:84-91."""
    return _join(["ID"] + ["Control1(1)"] * (n - 2) + ["Target1(Z)"])


def grover_iteration_steps(n, search_value):
    steps = [grover_oracle_step(n, search_value)]
    for q in range(1, n):
        steps.append(_single(n, q, "H"))
        steps.append(_single(n, q, "X"))
    steps.append(grover_controlled_z_step(n))
    for q in range(n - 1, 0, -1):
        steps.append(_single(n, q, "X"))
        steps.append(_single(n, q, "H"))
    return steps


def grover_reference_iterations(n):
    return int(math.pi / 4.0 * math.sqrt(1 << (n - 1)))


def grover_reference(n: int, search_value: int, iterations: int | None = None) -> CircuitSpec:
    """Grover() as grover.out runs it: n qubits, qubit 0 is the ancilla."""
    k = grover_reference_iterations(n) if iterations is None else iterations
    return CircuitSpec("grover_ref", n, 1 << (n - 1), {},
                       [([hadamard_step(n)], 1, True), (grover_iteration_steps(n, search_value), k, False)],
                       {"search_value": search_value, "iterations": k, "search_mask": (1 << (n - 1)) - 1})


def grover_search(m: int, w: int, iterations: int | None = None) -> CircuitSpec:
    """Ancilla-free Grover on m qubits, marked index w (index bit b <-> qubit m-1-b)."""
    k = int(math.pi / 4.0 * math.sqrt(1 << m)) if iterations is None else iterations
    gates = {"ZF1": [1, 0, 0, -1], "ZF0": [-1, 0, 0, 1]}
    # phase flip on |w>: controls on qubits 0..m-2 = bits m-1..1 of w,
    # target on qubit m-1 (bit 0) with diag(1,-1) if bit 0 of w is 1 else diag(-1,1)
    t = [""] * m
    for q in range(m - 1):
        bit = (w >> (m - 1 - q)) & 1
        t[q] = "Control1(1)" if bit else "Control1(0)"
    t[m - 1] = "Target1(ZF1)" if (w & 1) else "Target1(ZF0)"
    oracle = _join(t)
    z0 = _join(["Control1(0)"] * (m - 1) + ["Target1(ZF0)"])
    h = hadamard_step(m)
    return CircuitSpec("grover", m, 0, gates,
                       [([h], 1, True), ([oracle, h, z0, h], k, False)],
                       {"search_value": w, "iterations": k, "search_mask": (1 << m) - 1})


def rz(theta):
    return [np.exp(-0.5j * theta), 0.0, 0.0, np.exp(0.5j * theta)]


def ry(phi):
    c, s = math.cos(phi / 2.0), math.sin(phi / 2.0)
    return [c, -s, s, c]


def random_layered(n: int, layers: int, seed: int) -> CircuitSpec:
    rng = np.random.default_rng(seed)
    gates, steps = {}, []
    for layer in range(layers):
        theta = rng.uniform(0.0, 2.0 * math.pi, n)
        phi = rng.uniform(0.0, 2.0 * math.pi, n)
        rz_step, ry_step = [], []
        for q in range(n):
            a, b = f"rz{layer}_{q}", f"ry{layer}_{q}"
            gates[a] = rz(theta[q])
            gates[b] = ry(phi[q])
            rz_step.append(a)
            ry_step.append(b)
        steps.append(_join(rz_step))
        steps.append(_join(ry_step))
        perm = rng.permutation(n)
        t = _row(n)
        for g in range(n // 2):
            c, tq = int(perm[2 * g]), int(perm[2 * g + 1])
            t[c] = f"Control{g + 1}(1)"
            t[tq] = f"Target{g + 1}(X)"
        steps.append(_join(t))
    return CircuitSpec("layered", n, 0, gates, [(steps, 1, True)], {"layers": layers, "seed": seed})


def _cnot(n, c, t):
    s = _row(n)
    s[c] = "Control1(1)"
    s[t] = "Target1(X)"
    return _join(s)


def qft(n: int, x: int = 0) -> CircuitSpec:
    """QFT of the basis state |x> (x as an index, qubit 0 = most significant bit)."""
    gates, steps = {}, []
    for k in range(2, n + 1):
        gates[f"QR{k}"] = [1.0, 0.0, 0.0, np.exp(2j * math.pi / float(1 << k))]
    for j in range(n):
        steps.append(_single(n, j, "H"))
        for k in range(j + 1, n):
            s = _row(n)
            s[k] = "Control1(1)"
            s[j] = f"Target1(QR{k - j + 1})"
            steps.append(_join(s))
    for j in range(n // 2):
        a, b = j, n - 1 - j
        steps += [_cnot(n, a, b), _cnot(n, b, a), _cnot(n, a, b)]
    return CircuitSpec("qft", n, x, gates, [(steps, 1, True)], {"x": x})
