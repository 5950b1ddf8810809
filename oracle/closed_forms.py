"""Analytic states for the benchmark circuits (test oracle only).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  These pin the oracle
independently of any simulator:

* ``hadamard_all``   H on every qubit of |0...0>: every amplitude 2^{-n/2}
                     (the value src/algorithms/lib_general.cpp:44 prints and
                     tests/smoke_test.sh:70-76 checks).
* ``grover_search``  k Grover iterations on an N = 2^m search space with a
                     phase oracle on w and the diffusion H (I - 2|0><0|) H:
                     marked amplitude (-1)^k sin((2k+1)t), others
                     (-1)^k cos((2k+1)t)/sqrt(N-1), t = asin(N^{-1/2}).
* ``grover_reference_form``  the same tensored with the reference's ancilla
                     (qubit 0 = index bit n-1, prepared in |->,
                     src/algorithms/lib_grover.cpp:31).
* ``qft_basis``      textbook QFT (with reversal swaps) of |x>:
                     amplitude_y = e^{2 pi i x y / 2^n} / 2^{n/2}.
"""
from __future__ import annotations

import math

import numpy as np


def hadamard_all(n: int) -> np.ndarray:
    return np.full(1 << n, 2.0 ** (-n / 2.0), dtype=np.complex128)


def grover_amplitudes(m: int, k: int):
    N = float(1 << m)
    t = math.asin(1.0 / math.sqrt(N))
    sign = -1.0 if (k % 2) else 1.0
    return sign * math.sin((2 * k + 1) * t), sign * math.cos((2 * k + 1) * t) / math.sqrt(N - 1.0)


def grover_search(m: int, w: int, k: int) -> np.ndarray:
    marked, other = grover_amplitudes(m, k)
    s = np.full(1 << m, other, dtype=np.complex128)
    s[w] = marked
    return s


def grover_reference_form(n: int, w: int, k: int) -> np.ndarray:
    """n-qubit state of the reference Grover (ancilla on index bit n-1)."""
    search = grover_search(n - 1, w, k)
    inv = 1.0 / math.sqrt(2.0)
    return np.concatenate([search * inv, search * -inv])


def qft_basis(n: int, x: int) -> np.ndarray:
    N = 1 << n
    y = np.arange(N, dtype=np.float64)
    # reduce x*y mod N exactly before forming the angle
    prod = (np.arange(N, dtype=np.int64) * (x % N)) % N
    return np.exp(2j * math.pi * prod.astype(np.float64) / N) / math.sqrt(N)
