"""Host-side mirror of StateCraft's circuit model (core/.../quantum/).

Same names, argument meaning and validation messages as the reference:
``QuantumCircuit`` (QuantumCircuit.java:9-575), its sealed ``Operation`` records
(:362-574), the single-qubit gate classes and ``StateVector`` (StateVector.java:9-81).
The engine flattens these records into the ``sc_op`` array of the C ABI.
"""
from __future__ import annotations

import cmath
import math
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

# --------------------------------------------------------------------------
# single-qubit gates (SingleQubitGate.java, Hadamard.java, Pauli*.java, S*.java,
# MatrixSingleQubitGate.java)
# --------------------------------------------------------------------------


class SingleQubitGate:
    """A 2x2 complex matrix; element(row, col) like SingleQubitGate.element."""

    name = "gate"

    def __init__(self, m00: complex, m01: complex, m10: complex, m11: complex):
        self._m = (complex(m00), complex(m01), complex(m10), complex(m11))

    def element(self, row: int, col: int) -> complex:
        if row not in (0, 1) or col not in (0, 1):
            raise IndexError("row and column must be 0 or 1")
        return self._m[2 * row + col]

    def matrix(self) -> np.ndarray:
        return np.array(self._m, dtype=np.complex128).reshape(2, 2)

    def __repr__(self) -> str:
        return f"{self.name}{self._m}"


_INV_SQRT2 = 1.0 / math.sqrt(2.0)


class Hadamard(SingleQubitGate):
    name = "H"

    def __init__(self):
        super().__init__(_INV_SQRT2, _INV_SQRT2, _INV_SQRT2, -_INV_SQRT2)


class PauliX(SingleQubitGate):
    name = "X"

    def __init__(self):
        super().__init__(0, 1, 1, 0)


class PauliY(SingleQubitGate):
    name = "Y"

    def __init__(self):
        super().__init__(0, -1j, 1j, 0)


class PauliZ(SingleQubitGate):
    name = "Z"

    def __init__(self):
        super().__init__(1, 0, 0, -1)


class SGate(SingleQubitGate):
    name = "S"

    def __init__(self):
        super().__init__(1, 0, 0, 1j)


class SdgGate(SingleQubitGate):
    name = "Sdg"

    def __init__(self):
        super().__init__(1, 0, 0, -1j)


class MatrixSingleQubitGate(SingleQubitGate):
    def __init__(self, name: str, m00: complex, m01: complex, m10: complex, m11: complex):
        super().__init__(m00, m01, m10, m11)
        self.name = name


def _cis(angle: float) -> complex:
    return complex(math.cos(angle), math.sin(angle))


def rx(angle: float) -> MatrixSingleQubitGate:
    """OpenQasmCircuitParser.rotationX (OpenQasmCircuitParser.java:650-657)."""
    half = angle / 2.0
    c, s = math.cos(half), math.sin(half)
    return MatrixSingleQubitGate("rx", c, complex(0.0, -s), complex(0.0, -s), c)


def ry(angle: float) -> MatrixSingleQubitGate:
    """OpenQasmCircuitParser.rotationY (OpenQasmCircuitParser.java:659-665)."""
    half = angle / 2.0
    c, s = math.cos(half), math.sin(half)
    return MatrixSingleQubitGate("ry", c, -s, s, c)


def rz(angle: float) -> MatrixSingleQubitGate:
    """OpenQasmCircuitParser.rotationZ (OpenQasmCircuitParser.java:667-670)."""
    half = angle / 2.0
    return MatrixSingleQubitGate("rz", _cis(-half), 0, 0, _cis(half))


def u3(theta: float, phi: float, lam: float) -> MatrixSingleQubitGate:
    """OpenQasmCircuitParser.uGate (OpenQasmCircuitParser.java:672-680)."""
    c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
    cl, cp, cpl = _cis(lam), _cis(phi), _cis(phi + lam)
    m01 = complex(cl.real * -s, cl.imag * -s)
    m10 = complex(cp.real * s, cp.imag * s)
    m11 = complex(cpl.real * c, cpl.imag * c)
    return MatrixSingleQubitGate("u", c, m01, m10, m11)


def zz_phase(gamma: float) -> list[complex]:
    """exp(-i gamma Z Z) diagonal (AlgorithmSuiteSpecs.java:283-287)."""
    aligned, anti = _cis(-gamma), _cis(gamma)
    return [aligned, anti, anti, aligned]


def rzz_diagonal(gamma: float) -> list[complex]:
    """RZZ(gamma) = exp(-i gamma/2 Z Z)."""
    return zz_phase(gamma / 2.0)


class CnotGate:
    """Marker gate (CnotGate.java)."""

    _instance = None

    @classmethod
    def of(cls) -> "CnotGate":
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance


# --------------------------------------------------------------------------
# operations (QuantumCircuit.Operation, QuantumCircuit.java:362-574)
# --------------------------------------------------------------------------


class Operation:
    def validate_targets(self, qubit_count: int) -> None:  # pragma: no cover - abstract
        raise NotImplementedError

    def qubits_touched(self) -> tuple[int, ...]:  # pragma: no cover - abstract
        raise NotImplementedError


def _require_non_negative(value: int, message: str) -> None:
    if value < 0:
        raise ValueError(message)


@dataclass(frozen=True)
class SingleGateOperation(Operation):
    gate: SingleQubitGate
    qubit: int

    def __post_init__(self):
        if self.gate is None:
            raise TypeError("gate")
        _require_non_negative(self.qubit, "qubit index must be non-negative")

    def validate_targets(self, qubit_count: int) -> None:
        if self.qubit >= qubit_count:
            raise ValueError(f"target qubit out of range: {self.qubit}")

    def qubits_touched(self):
        return (self.qubit,)


@dataclass(frozen=True)
class CnotOperation(Operation):
    gate: CnotGate
    controlQubit: int
    targetQubit: int

    def __post_init__(self):
        _require_non_negative(self.controlQubit, "control qubit index must be non-negative")
        _require_non_negative(self.targetQubit, "target qubit index must be non-negative")
        if self.controlQubit == self.targetQubit:
            raise ValueError("control and target qubits must differ")

    def validate_targets(self, qubit_count: int) -> None:
        if self.controlQubit >= qubit_count:
            raise ValueError(f"control qubit out of range: {self.controlQubit}")
        if self.targetQubit >= qubit_count:
            raise ValueError(f"target qubit out of range: {self.targetQubit}")

    def qubits_touched(self):
        return (self.controlQubit, self.targetQubit)


def _two_qubit_checks(first: int, second: int, same_message: str) -> None:
    if first < 0 or second < 0:
        raise ValueError("qubit indices must be non-negative")
    if first == second:
        raise ValueError(same_message)


def _range_checks(first: int, second: int, qubit_count: int) -> None:
    if first >= qubit_count:
        raise ValueError(f"first qubit out of range: {first}")
    if second >= qubit_count:
        raise ValueError(f"second qubit out of range: {second}")


@dataclass(frozen=True)
class TwoQubitGateOperation(Operation):
    matrix: tuple
    firstQubit: int
    secondQubit: int

    def __post_init__(self):
        if len(self.matrix) != 16:
            raise ValueError("matrix must contain 16 elements")
        _two_qubit_checks(self.firstQubit, self.secondQubit, "qubits must be distinct")

    def validate_targets(self, qubit_count: int) -> None:
        _range_checks(self.firstQubit, self.secondQubit, qubit_count)

    def qubits_touched(self):
        return (self.firstQubit, self.secondQubit)


@dataclass(frozen=True)
class TwoQubitDiagonalOperation(Operation):
    diagonal: tuple
    firstQubit: int
    secondQubit: int

    def __post_init__(self):
        if len(self.diagonal) != 4:
            raise ValueError("diagonal must contain 4 elements")
        _two_qubit_checks(self.firstQubit, self.secondQubit, "qubits must be distinct")

    def validate_targets(self, qubit_count: int) -> None:
        _range_checks(self.firstQubit, self.secondQubit, qubit_count)

    def qubits_touched(self):
        return (self.firstQubit, self.secondQubit)


@dataclass(frozen=True)
class SwapOperation(Operation):
    firstQubit: int
    secondQubit: int

    def __post_init__(self):
        _two_qubit_checks(self.firstQubit, self.secondQubit, "cannot swap qubit with itself")

    def validate_targets(self, qubit_count: int) -> None:
        _range_checks(self.firstQubit, self.secondQubit, qubit_count)

    def qubits_touched(self):
        return (self.firstQubit, self.secondQubit)


@dataclass(frozen=True)
class MultiControlOperation(Operation):
    gate: SingleQubitGate
    targetQubit: int
    controlQubits: tuple

    def __post_init__(self):
        controls = tuple(sorted(self.controlQubits))
        object.__setattr__(self, "controlQubits", controls)
        _require_non_negative(self.targetQubit, "target qubit index must be non-negative")
        if not controls:
            raise ValueError("at least one control qubit is required")
        for c in controls:
            _require_non_negative(c, "control qubit index must be non-negative")
            if c == self.targetQubit:
                raise ValueError("control and target qubits must differ")
        for a, b in zip(controls, controls[1:]):
            if a == b:
                raise ValueError(f"duplicate control qubit: {b}")

    def validate_targets(self, qubit_count: int) -> None:
        if self.targetQubit >= qubit_count:
            raise ValueError(f"target qubit out of range: {self.targetQubit}")
        for c in self.controlQubits:
            if c >= qubit_count:
                raise ValueError(f"control qubit out of range: {c}")

    def qubits_touched(self):
        return (self.targetQubit,) + tuple(self.controlQubits)


@dataclass(frozen=True)
class MeasureOperation(Operation):
    qubits: tuple

    def __post_init__(self):
        if not self.qubits:
            raise ValueError("at least one qubit must be measured")
        qs = tuple(sorted(self.qubits))
        for q in qs:
            _require_non_negative(q, "measured qubit index must be non-negative")
        for a, b in zip(qs, qs[1:]):
            if a == b:
                raise ValueError(f"duplicate measured qubit: {b}")
        object.__setattr__(self, "qubits", qs)

    def validate_targets(self, qubit_count: int) -> None:
        for q in self.qubits:
            if q >= qubit_count:
                raise ValueError(f"measured qubit out of range: {q}")

    def qubits_touched(self):
        return tuple(self.qubits)


# --------------------------------------------------------------------------
# QuantumCircuit
# --------------------------------------------------------------------------


@dataclass(frozen=True)
class QuantumCircuit:
    """Immutable circuit; every append returns a new circuit (QuantumCircuit.java:29-100)."""

    qubitCount: int
    operations: tuple = field(default_factory=tuple)

    def __post_init__(self):
        if self.qubitCount <= 0:
            raise ValueError("qubitCount must be positive")
        ops = tuple(self.operations)
        for op in ops:
            if op is None:
                raise TypeError("operation")
            op.validate_targets(self.qubitCount)
        object.__setattr__(self, "operations", ops)

    # builder API -------------------------------------------------------------
    def _append(self, op: Operation) -> "QuantumCircuit":
        op.validate_targets(self.qubitCount)
        return QuantumCircuit(self.qubitCount, self.operations + (op,))

    def append(self, gate, *qubits: int) -> "QuantumCircuit":
        if isinstance(gate, CnotGate):
            control, target = qubits
            return self._append(CnotOperation(gate, control, target))
        (target,) = qubits
        return self._append(SingleGateOperation(gate, target))

    def appendTwoQubitUnitary(self, matrix: Sequence[complex], first: int, second: int):
        if len(matrix) != 16:
            raise ValueError("two-qubit matrix must contain 16 elements")
        return self._append(TwoQubitGateOperation(tuple(complex(x) for x in matrix), first, second))

    def appendDiagonalTwoQubit(self, diagonal: Sequence[complex], first: int, second: int):
        if len(diagonal) != 4:
            raise ValueError("two-qubit diagonal must contain 4 elements")
        return self._append(
            TwoQubitDiagonalOperation(tuple(complex(x) for x in diagonal), first, second))

    def appendControlledPhase(self, angle: float, control: int, target: int):
        phase = complex(math.cos(angle), math.sin(angle))
        return self.appendDiagonalTwoQubit([1, 1, 1, phase], control, target)

    def appendControlled(self, gate: SingleQubitGate, control: int, target: int):
        return self.appendMultiControl(gate, target, control)

    def appendControlledX(self, control: int, target: int):
        return self.appendControlled(PauliX(), control, target)

    def appendControlledY(self, control: int, target: int):
        return self.appendControlled(PauliY(), control, target)

    def appendControlledZ(self, control: int, target: int):
        return self.appendControlled(PauliZ(), control, target)

    def appendToffoli(self, c0: int, c1: int, target: int):
        return self.appendMultiControl(PauliX(), target, c0, c1)

    def appendSwap(self, first: int, second: int):
        return self._append(SwapOperation(first, second))

    def appendMultiControl(self, gate: SingleQubitGate, target: int, *controls: int):
        if not controls:
            raise ValueError("at least one control qubit is required")
        cs = sorted(controls)
        for c in cs:
            if c < 0:
                raise ValueError("control qubit index must be non-negative")
        for a, b in zip(cs, cs[1:]):
            if a == b:
                raise ValueError(f"duplicate control qubit: {b}")
        return self._append(MultiControlOperation(gate, target, tuple(cs)))

    def measure(self, *qubits: int):
        return self._append(MeasureOperation(tuple(qubits)))


# --------------------------------------------------------------------------
# StateVector (StateVector.java:9-81)
# --------------------------------------------------------------------------


class StateVector:
    """Interleaved (re, im) amplitudes, little-endian qubit order."""

    MAX_DENSE_QUBITS = 29  # StateVector.java:11 (Java array limit)

    def __init__(self, qubit_count: int, data: np.ndarray):
        self._n = qubit_count
        self._data = data

    @staticmethod
    def fromArray(qubit_count: int, data) -> "StateVector":
        if qubit_count <= 0:
            raise ValueError("qubitCount must be positive")
        if qubit_count > StateVector.MAX_DENSE_QUBITS:
            raise NotImplementedError(
                f"dense state vectors support up to {StateVector.MAX_DENSE_QUBITS} qubits")
        arr = np.array(data, dtype=np.float64, copy=True).reshape(-1)
        expected = 2 << qubit_count
        if arr.size != expected:
            raise ValueError(f"Expected data length {expected}, got {arr.size}")
        return StateVector(qubit_count, arr)

    def qubitCount(self) -> int:
        return self._n

    def dimension(self) -> int:
        return 1 << self._n

    def data(self) -> np.ndarray:
        return self._data.copy()

    def copyData(self) -> np.ndarray:
        return self._data.copy()

    def real(self, index: int) -> float:
        return float(self._data[2 * index])

    def imag(self, index: int) -> float:
        return float(self._data[2 * index + 1])

    def amplitudes(self) -> np.ndarray:
        return self._data.view(np.complex128)


def cmath_phase(angle: float) -> complex:
    return cmath.exp(1j * angle)
