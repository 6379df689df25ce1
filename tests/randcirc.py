"""Seeded random circuits covering every operation kind and gate shape the engine
special-cases (dense / diagonal / X-like single gates, controlled and multi-controlled
gates, dense and diagonal two-qubit unitaries, swaps)."""
from __future__ import annotations

import numpy as np

from statecraft_b200 import quantum as Q


def random_unitary(rng: np.random.Generator, dim: int) -> np.ndarray:
    z = (rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def random_gate(rng) -> Q.SingleQubitGate:
    k = rng.integers(0, 6)
    if k == 0:
        return Q.PauliX()
    if k == 1:
        return Q.rz(float(rng.uniform(0, 2 * np.pi)))  # diagonal
    if k == 2:
        return Q.Hadamard()
    u = random_unitary(rng, 2)
    return Q.MatrixSingleQubitGate("u", u[0, 0], u[0, 1], u[1, 0], u[1, 1])


def random_circuit(n: int, depth: int, seed: int, kinds=None) -> Q.QuantumCircuit:
    rng = np.random.default_rng(seed)
    c = Q.QuantumCircuit(n)
    kinds = kinds or ["single", "cnot", "two", "diag2", "swap", "multi", "cphase"]
    for _ in range(depth):
        kind = kinds[rng.integers(0, len(kinds))]
        if n < 2 and kind != "single":
            kind = "single"
        qs = rng.permutation(n)
        if kind == "single":
            c = c.append(random_gate(rng), int(qs[0]))
        elif kind == "cnot":
            c = c.append(Q.CnotGate.of(), int(qs[0]), int(qs[1]))
        elif kind == "two":
            if rng.random() < 0.3:
                d = np.exp(1j * rng.uniform(0, 2 * np.pi, 4))
                m = np.diag(d)
            else:
                m = random_unitary(rng, 4)
            c = c.appendTwoQubitUnitary(list(m.reshape(-1)), int(qs[0]), int(qs[1]))
        elif kind == "diag2":
            d = np.exp(1j * rng.uniform(0, 2 * np.pi, 4))
            c = c.appendDiagonalTwoQubit(list(d), int(qs[0]), int(qs[1]))
        elif kind == "swap":
            c = c.appendSwap(int(qs[0]), int(qs[1]))
        elif kind == "cphase":
            c = c.appendControlledPhase(float(rng.uniform(0, 2 * np.pi)), int(qs[0]), int(qs[1]))
        elif kind == "multi":
            nc = int(rng.integers(1, min(n - 1, 4) + 1))
            c = c.appendMultiControl(random_gate(rng), int(qs[0]), *[int(x) for x in qs[1:1 + nc]])
    return c


def random_state(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    a /= np.linalg.norm(a)
    out = np.empty(2 << n)
    out[0::2], out[1::2] = a.real, a.imag
    return out
