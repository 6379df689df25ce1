"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Every random draw comes from a SplitMix64 stream (java.util.SplittableRandom's
generator), so a Java caller can rebuild the identical circuits:

- ``brickwall_circuit``: U3(theta, phi, lambda) on every qubit per layer, angles
  drawn layer -> qubit -> (theta, phi, lambda) as nextDouble(2*pi); then CNOT(i, i+1)
  for even i on even layers and odd i on odd layers; optionally a multi-controlled Z
  on the all-ones pattern (target n-1, controls 0..n-2) and RZZ(gamma) =
  exp(-i gamma/2 Z Z) on a random pair.  20 qubits x 20 layers (seed 2020) and
  30 qubits x 40 layers with MCZ + RZZ (seed 3030) are the plain-drop-in configs.
- ``qaoa_instances``: ring-QAOA parameters for batched runs.
- ``hea_ansatz`` / ``random_pauli_sum``: the adjoint-gradient workload.
- ``ghz_circuit``: H + CNOT chain for the noisy-trajectory workload.
Gate conventions: core/.../parse/OpenQasmCircuitParser.java:650-684,
app/.../AlgorithmSuiteSpecs.java:283-300.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from . import quantum as Q

TWO_PI = 2.0 * math.pi
_GAMMA = 0x9E3779B97F4A7C15
_M64 = 0xFFFFFFFFFFFFFFFF


class SplitMix64:
    """java.util.SplittableRandom(seed): nextLong / nextDouble / nextDouble(bound)."""

    def __init__(self, seed: int):
        self.state = seed & _M64

    def nextLong(self) -> int:
        self.state = (self.state + _GAMMA) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def nextDouble(self, bound: float | None = None) -> float:
        r = (self.nextLong() >> 11) * 2.0 ** -53
        if bound is None:
            return r
        r *= bound
        return r if r < bound else math.nextafter(bound, -math.inf)

    def nextIndex(self, bound: int) -> int:
        """floor(nextDouble() * bound), clamped to bound - 1."""
        return min(bound - 1, int(self.nextDouble() * bound))

    def nextGaussian(self) -> float:
        """Box-Muller on two nextDouble() draws."""
        u1 = self.nextDouble()
        u2 = self.nextDouble()
        return math.sqrt(-2.0 * math.log1p(-u1)) * math.cos(TWO_PI * u2)


def brickwall_circuit(n: int, layers: int, seed: int, mcz: bool = False,
                      rzz: bool = False) -> Q.QuantumCircuit:
    rng = SplitMix64(seed)
    ops = []
    for layer in range(layers):
        for q in range(n):
            th, ph, la = rng.nextDouble(TWO_PI), rng.nextDouble(TWO_PI), rng.nextDouble(TWO_PI)
            ops.append(Q.SingleGateOperation(Q.u3(th, ph, la), q))
        for i in range(layer % 2, n - 1, 2):
            ops.append(Q.CnotOperation(Q.CnotGate.of(), i, i + 1))
        if mcz:
            ops.append(Q.MultiControlOperation(Q.PauliZ(), n - 1, tuple(range(n - 1))))
        if rzz:
            i = rng.nextIndex(n)
            j = rng.nextIndex(n - 1)
            if j >= i:
                j += 1
            gamma = rng.nextDouble(TWO_PI)
            ops.append(Q.TwoQubitDiagonalOperation(tuple(Q.rzz_diagonal(gamma)), i, j))
    return Q.QuantumCircuit(n, tuple(ops))


def amp_updates(circuit: Q.QuantumCircuit) -> float:
    """Gate-level amplitude updates: dense 1q/2q and diagonal gates count 2^n,
    CNOT and SWAP 2^(n-1), a gate with c controls 2^(n-c)."""
    n = circuit.qubitCount
    total = 0.0
    for op in circuit.operations:
        if isinstance(op, (Q.CnotOperation, Q.SwapOperation)):
            total += 2.0 ** (n - 1)
        elif isinstance(op, Q.MultiControlOperation):
            total += 2.0 ** (n - len(op.controlQubits))
        elif isinstance(op, Q.MeasureOperation):
            continue
        else:
            total += 2.0 ** n
    return total


def dense_window_circuit(n: int, depth: int, seed: int) -> Q.QuantumCircuit:
    """Hadamards, then `depth` rounds of 12 gates inside a random 5-qubit window:
    dense random two-qubit unitaries, CNOTs, random single-qubit gates and
    controlled phases; every third round ends with a multi-controlled Z on all
    qubits.  Runs of gates on at most 5 qubits with much dense work: the shape the
    tensor-core blocks are for."""
    rng = np.random.default_rng(seed)
    c = Q.QuantumCircuit(n)
    for q in range(n):
        c = c.append(Q.Hadamard(), q)
    for d in range(depth):
        lo = int(rng.integers(0, n - 4))
        for _ in range(12):
            a, b = (int(x) + lo for x in rng.choice(5, 2, replace=False))
            kind = int(rng.integers(0, 4))
            if kind == 0:
                z = (rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))) / np.sqrt(2)
                qm, r = np.linalg.qr(z)
                m = qm * (np.diag(r) / np.abs(np.diag(r)))
                c = c.appendTwoQubitUnitary(list(m.reshape(-1)), a, b)
            elif kind == 1:
                c = c.append(Q.CnotGate.of(), a, b)
            elif kind == 2:
                th, ph, la = rng.uniform(0, TWO_PI, 3)
                c = c.append(Q.u3(float(th), float(ph), float(la)), a)
            else:
                c = c.appendControlledPhase(float(rng.uniform(0, TWO_PI)), a, b)
        if d % 3 == 2:
            c = c.appendMultiControl(Q.PauliZ(), n - 1, *range(n - 1))
    return c


# ---------------------------------------------------------------------------
# batched QAOA
# ---------------------------------------------------------------------------
@dataclass
class QaoaBatch:
    n_qubits: np.ndarray  # int32 [instances]
    gammas: np.ndarray    # float64 [instances, p]
    betas: np.ndarray     # float64 [instances, p]

    @property
    def instances(self) -> int:
        return int(self.n_qubits.size)

    @property
    def p(self) -> int:
        return int(self.gammas.shape[1])


def qaoa_instances(count: int, p: int, seed: int, n_min: int = 10, n_max: int = 22) -> QaoaBatch:
    """n_i ~ U{n_min..n_max}; gamma_l, beta_l ~ U[0, pi) per instance."""
    rng = SplitMix64(seed)
    nq = np.empty(count, dtype=np.int32)
    g = np.empty((count, p))
    b = np.empty((count, p))
    for i in range(count):
        nq[i] = n_min + rng.nextIndex(n_max - n_min + 1)
        for layer in range(p):
            g[i, layer] = rng.nextDouble(math.pi)
            b[i, layer] = rng.nextDouble(math.pi)
    return QaoaBatch(nq, g, b)


def qaoa_circuit(n: int, gammas, betas) -> Q.QuantumCircuit:
    """H on all qubits, then per layer exp(-i g Z_i Z_{i+1 mod n}) on the ring and RX(2b)
    (AlgorithmSuiteSpecs.qaoaRingAnsatz, AlgorithmSuiteSpecs.java:186-200)."""
    c = Q.QuantumCircuit(n)
    for q in range(n):
        c = c.append(Q.Hadamard(), q)
    for g, b in zip(gammas, betas):
        for q in range(n):
            c = c.appendDiagonalTwoQubit(Q.zz_phase(float(g)), q, (q + 1) % n)
        for q in range(n):
            c = c.append(Q.rx(2.0 * float(b)), q)
    return c


# ---------------------------------------------------------------------------
# adjoint workload
# ---------------------------------------------------------------------------
def hea_ops(n: int, layers: int):
    """Hardware-efficient ansatz as sc_op records: per layer RY(theta) and RZ(theta) on
    every qubit (one parameter each) then a CNOT ring i -> i+1 mod n."""
    ops = []
    p = 0
    for _ in range(layers):
        for q in range(n):
            ops.append((A.SC_OP_RY, q, -1, p))
            p += 1
        for q in range(n):
            ops.append((A.SC_OP_RZ, q, -1, p))
            p += 1
        for q in range(n):
            ops.append((A.SC_OP_CNOT, q, (q + 1) % n, -1))
    arr = (A.ScOp * len(ops))()
    for i, (kind, q0, q1, param) in enumerate(ops):
        arr[i].kind, arr[i].q0, arr[i].q1, arr[i].param = kind, q0, q1, param
    return arr, len(ops), p


def hea_params(count: int, seed: int) -> np.ndarray:
    rng = SplitMix64(seed)
    return np.array([rng.nextDouble(TWO_PI) for _ in range(count)])


def random_pauli_sum(n: int, terms: int, seed: int):
    """c_k ~ N(0, 1); each qubit of P_k uniform over I, X, Y, Z.  Returns (x, z, c)."""
    rng = SplitMix64(seed)
    x = np.zeros(terms, dtype=np.uint64)
    z = np.zeros(terms, dtype=np.uint64)
    c = np.zeros(terms)
    for k in range(terms):
        c[k] = rng.nextGaussian()
        xm = zm = 0
        for q in range(n):
            letter = rng.nextIndex(4)  # 0 I, 1 X, 2 Y, 3 Z
            if letter in (1, 2):
                xm |= 1 << q
            if letter in (2, 3):
                zm |= 1 << q
        x[k], z[k] = xm, zm
    return x, z, c


# ---------------------------------------------------------------------------
# noisy GHZ
# ---------------------------------------------------------------------------
def ghz_circuit(n: int) -> Q.QuantumCircuit:
    c = Q.QuantumCircuit(n).append(Q.Hadamard(), 0)
    for i in range(n - 1):
        c = c.append(Q.CnotGate.of(), i, i + 1)
    return c
