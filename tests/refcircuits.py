"""The reference's statevector test cases, rebuilt with the host API.

Each builder returns a SimulationRequest plus the naive expected amplitudes the
reference test compares against (QuantumCircuit.apply, 1e-12).  Sources:
engines/src/test/java/com/omaarr90/statecraft/engines/statevector/StatevectorEngineTest.java
(cited per case).  Random circuits/states use the same generators and seeds as
the JUnit tests (java.util.Random / SplittableRandom restatements).
"""
from __future__ import annotations

import math

import numpy as np

from java_random import JavaRandom
from oracle import naive
from oracle import oracle as O
from statecraft_b200 import quantum as Q
from statecraft_b200.engine import SimulationRequest

RANDOM_SEED = 0x51D5  # StatevectorEngineTest.java:30


def _random_single_gate(r: JavaRandom) -> Q.SingleQubitGate:
    # randomSingleGate (StatevectorEngineTest.java:442-449)
    return (Q.PauliX, Q.PauliY, Q.PauliZ, Q.Hadamard)[r.nextInt(4)]()


def _random_two_qubit_circuit(r: JavaRandom, depth: int) -> Q.QuantumCircuit:
    # randomTwoQubitCircuit (StatevectorEngineTest.java:428-440)
    c = Q.QuantumCircuit(2)
    for _ in range(depth):
        if r.nextBoolean():
            g = _random_single_gate(r)
            c = c.append(g, r.nextInt(2))
        else:
            control = r.nextInt(2)
            c = c.append(Q.CnotGate.of(), control, 1 - control)
    return c


def _extract_unitary(c: Q.QuantumCircuit) -> list[complex]:
    # extractUnitaryMatrix (StatevectorEngineTest.java:451-463)
    dim = 1 << c.qubitCount
    m = [0j] * (dim * dim)
    for col in range(dim):
        basis = [0j] * dim
        basis[col] = 1 + 0j
        out = naive.apply(c, basis)
        for row in range(dim):
            m[row * dim + col] = out[row]
    return m


def _random_normalized_state(r: JavaRandom, dim: int) -> list[complex]:
    # randomNormalizedState (StatevectorEngineTest.java:465-478)
    st = []
    nsq = 0.0
    for _ in range(dim):
        re = r.nextDouble() - 0.5
        im = r.nextDouble() - 0.5
        st.append(complex(re, im))
        nsq += re * re + im * im
    scale = 1.0 / math.sqrt(nsq)
    return [complex(a.real * scale, a.imag * scale) for a in st]


def _to_state_vector(n: int, amps: list[complex]) -> Q.StateVector:
    data = np.empty(2 << n)
    data[0::2] = [a.real for a in amps]
    data[1::2] = [a.imag for a in amps]
    return Q.StateVector.fromArray(n, data)


def _qft(n: int) -> Q.QuantumCircuit:
    # buildQftCircuit (StatevectorEngineTest.java:480-494)
    c = Q.QuantumCircuit(n)
    for t in range(n):
        c = c.append(Q.Hadamard(), t)
        for ctl in range(t + 1, n):
            c = c.appendControlledPhase(math.pi / (1 << (ctl - t)), ctl, t)
    for i in range(n // 2):
        c = c.appendSwap(i, n - i - 1)
    return c


def cases():
    """(name, request, expected amplitudes as complex list)."""
    out = []
    # simulateFromZeroStateMatchesCircuitApply (:38-47)
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
    out.append(("bell", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateFromCustomStateMatchesCircuitApply (:49-60)
    c = Q.QuantumCircuit(1).append(Q.Hadamard(), 0)
    init = Q.StateVector.fromArray(1, [0.0, 0.0, 1.0, 0.0])
    out.append(("custom_state", SimulationRequest.withInitialState(c, init), naive.apply(c, [0j, 1 + 0j])))
    # simulateFromBasisStateMatchesCircuitApply (:62-73)
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 1).append(Q.PauliZ(), 0)
    out.append(("basis_state", SimulationRequest.zeroState(c).withBasisState(0),
                naive.apply(c, [0j, 1 + 0j, 0j, 0j])))
    # simulateIdentityCircuitPreservesInitialStateAmplitudes (:75-104)
    rng = O.SplittableRandom(RANDOM_SEED ^ 0x5151)
    data = []
    nsq = 0.0
    for _ in range(8):
        re = rng.nextDouble() - 0.5
        im = rng.nextDouble() - 0.5
        data += [re, im]
        nsq += re * re + im * im
    s = 1.0 / math.sqrt(nsq)
    data = [x * s for x in data]
    init = Q.StateVector.fromArray(3, data)
    out.append(("identity", SimulationRequest.withInitialState(Q.QuantumCircuit(3), init),
                [complex(data[2 * k], data[2 * k + 1]) for k in range(8)]))
    # simulateMultiQubitCircuitMatchesReference (:106-116)
    c = (Q.QuantumCircuit(5).append(Q.Hadamard(), 4).append(Q.Hadamard(), 1).append(Q.PauliX(), 0)
         .append(Q.CnotGate.of(), 4, 2).append(Q.Hadamard(), 2))
    out.append(("multi_qubit", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateTwoQubitUnitaryMatchesReference (:124-133)
    r = JavaRandom(RANDOM_SEED)
    for trial in range(6):
        m = _extract_unitary(_random_two_qubit_circuit(r, 6))
        c = Q.QuantumCircuit(2).appendTwoQubitUnitary(m, 0, 1)
        out.append((f"two_qubit_unitary_{trial}", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateTwoQubitUnitaryOnNonAdjacentQubitsMatchesReference (:135-146)
    r = JavaRandom(RANDOM_SEED ^ 0x8FF0)
    m = _extract_unitary(_random_two_qubit_circuit(r, 5))
    c = (Q.QuantumCircuit(3).append(Q.Hadamard(), 1).appendTwoQubitUnitary(m, 2, 0)
         .append(Q.PauliZ(), 1))
    out.append(("two_qubit_nonadjacent", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateControlledPhaseMatchesReference (:148-159)
    for lo_first in (True, False):
        c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.Hadamard(), 1)
        c = c.appendControlledPhase(math.pi / 3.0, 0, 1) if lo_first else c.appendControlledPhase(math.pi / 3.0, 1, 0)
        out.append((f"controlled_phase_{int(lo_first)}", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateSwapMatchesReference (:161-169)
    c = (Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.PauliX(), 2).appendSwap(0, 2)
         .append(Q.Hadamard(), 1))
    out.append(("swap", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateMultiControlMatchesReference (:171-178) and three controls (:180-188)
    c = Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.Hadamard(), 1).appendMultiControl(Q.PauliX(), 2, 0, 1)
    out.append(("multi_control_2", SimulationRequest.zeroState(c), naive.apply(c)))
    c = (Q.QuantumCircuit(4).append(Q.Hadamard(), 0).append(Q.Hadamard(), 1).append(Q.Hadamard(), 2)
         .appendMultiControl(Q.PauliX(), 3, 0, 1, 2))
    out.append(("multi_control_3", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateGhZCircuitMatchesReference (:190-197)
    c = (Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
         .appendMultiControl(Q.PauliX(), 2, 0, 1))
    out.append(("ghz", SimulationRequest.zeroState(c), naive.apply(c)))
    # simulateQftThreeQubitsMatchesReference (:199-211)
    r = JavaRandom(RANDOM_SEED ^ 0xABCD)
    init = _random_normalized_state(r, 8)
    qft = _qft(3)
    out.append(("qft3", SimulationRequest.withInitialState(qft, _to_state_vector(3, init)),
                naive.apply(qft, init)))
    # parallelExecutionMatchesSerialForMixedStatevectorOperations (:213-235): circuit only
    r = JavaRandom(RANDOM_SEED ^ 0xFACEB00C)
    m = _extract_unitary(_random_two_qubit_circuit(r, 7))
    c = (Q.QuantumCircuit(6).append(_random_single_gate(r), 0).append(_random_single_gate(r), 5)
         .append(Q.CnotGate.of(), 5, 1).appendSwap(0, 4).appendTwoQubitUnitary(m, 5, 2)
         .appendControlledPhase(math.pi / 7.0, 4, 3).appendMultiControl(Q.PauliY(), 1, 0, 2, 5)
         .append(_random_single_gate(r), 3))
    init = _random_normalized_state(r, 64)
    out.append(("mixed_6q", SimulationRequest.withInitialState(c, _to_state_vector(6, init)),
                naive.apply(c, init)))
    return out


def large_basis_case():
    """largeCircuitNearTargetLimitRemainsNumericallySane (:365-379): 22-qubit KAT."""
    c = (Q.QuantumCircuit(22).append(Q.PauliX(), 0).append(Q.PauliX(), 5).append(Q.PauliX(), 21)
         .append(Q.CnotGate.of(), 21, 1).append(Q.CnotGate.of(), 0, 2).appendSwap(5, 3))
    expected_index = (1 << 0) | (1 << 1) | (1 << 2) | (1 << 3) | (1 << 21)
    return SimulationRequest.zeroState(c), expected_index


def to_interleaved(amps: list[complex]) -> np.ndarray:
    a = np.asarray(amps, dtype=np.complex128)
    out = np.empty(2 * a.size)
    out[0::2] = a.real
    out[1::2] = a.imag
    return out
