"""Host-side mirror of StateCraft's noise model (core/.../core/noise/).

``ErrorChannel`` factories build the same Kraus operators as the reference
channel classes; ``NoiseModel.scheduledChannelsAfter`` returns channels in the
reference order (NoiseModel.java:211-241): gate-type channels, then idle channels
on untouched qubits (in java.util.HashMap iteration order), then global channels.
``flatten_schedule`` turns a circuit + model into the ``sc_channel`` records the
C ABI consumes, visiting composites and targets like
StatevectorEngine.applyErrorChannel (StatevectorEngine.java:382-407).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import quantum as Q


class KrausOperator:
    def __init__(self, matrix: Sequence[complex]):
        m = tuple(complex(x) for x in matrix)
        dim = int(math.isqrt(len(m)))
        if not m:
            raise ValueError("matrix must not be empty")
        if dim * dim != len(m):
            raise ValueError(f"matrix length must be a perfect square, got {len(m)}")
        self.matrix = m
        self.dimension = dim
        self.numQubits = dim.bit_length() - 1


class ErrorChannel:
    """Sealed channel interface (ErrorChannel.java)."""

    def krausDecomposition(self) -> list[KrausOperator]:  # pragma: no cover - abstract
        raise NotImplementedError

    def affectedQubits(self) -> tuple[int, ...]:  # pragma: no cover - abstract
        raise NotImplementedError

    # factories (ErrorChannel.java:42-130)
    @staticmethod
    def depolarizing(probability: float, *qubits: int) -> "ErrorChannel":
        return DepolarizingChannel(probability, qubits)

    @staticmethod
    def amplitudeDamping(gamma: float, *qubits: int) -> "ErrorChannel":
        return AmplitudeDampingChannel(gamma, qubits)

    @staticmethod
    def phaseFlip(probability: float, *qubits: int) -> "ErrorChannel":
        return PhaseFlipChannel(probability, qubits)

    @staticmethod
    def phaseDamping(lam: float, *qubits: int) -> "ErrorChannel":
        return PhaseDampingChannel(lam, qubits)

    @staticmethod
    def thermalRelaxation(t1: float, t2: float, gate_time: float, *qubits: int) -> "ErrorChannel":
        return ThermalRelaxationChannel(t1, t2, gate_time, qubits)

    @staticmethod
    def compose(*channels: "ErrorChannel") -> "ErrorChannel":
        return CompositeChannel(channels)


class _SingleQubitChannel(ErrorChannel):
    kind = "channel"

    def __init__(self, qubits: Sequence[int]):
        if len(qubits) != 1:
            raise ValueError(f"{self.kind} channel currently only supports single qubits")
        self._qubits = tuple(int(q) for q in qubits)

    def affectedQubits(self):
        return self._qubits


def _check_unit(name: str, value: float) -> None:
    if value < 0.0 or value > 1.0 or math.isnan(value):
        raise ValueError(f"{name} must be in [0,1], got {value}")


class DepolarizingChannel(_SingleQubitChannel):
    """DepolarizingChannel.java:49-76: K0 = sqrt(1-p) I, K1..3 = sqrt(p/3) {X, Y, Z}."""

    kind = "depolarizing"

    def __init__(self, probability: float, qubits):
        _check_unit("probability", probability)
        super().__init__(qubits)
        self.probability = probability

    def krausDecomposition(self):
        p = self.probability
        a = math.sqrt(1.0 - p)
        b = math.sqrt(p / 3.0)
        return [KrausOperator([a, 0, 0, a]),
                KrausOperator([0, b, b, 0]),
                KrausOperator([0, complex(0.0, -b), complex(0.0, b), 0]),
                KrausOperator([b, 0, 0, -b])]


class AmplitudeDampingChannel(_SingleQubitChannel):
    """AmplitudeDampingChannel.java:47-61."""

    kind = "amplitude damping"

    def __init__(self, gamma: float, qubits):
        _check_unit("gamma", gamma)
        super().__init__(qubits)
        self.gamma = gamma

    def krausDecomposition(self):
        g = self.gamma
        return [KrausOperator([1, 0, 0, math.sqrt(1.0 - g)]),
                KrausOperator([0, math.sqrt(g), 0, 0])]


class PhaseFlipChannel(_SingleQubitChannel):
    """PhaseFlipChannel.java:50-63."""

    kind = "phase flip"

    def __init__(self, probability: float, qubits):
        _check_unit("probability", probability)
        super().__init__(qubits)
        self.probability = probability

    def krausDecomposition(self):
        p = self.probability
        a, b = math.sqrt(1.0 - p), math.sqrt(p)
        return [KrausOperator([a, 0, 0, a]), KrausOperator([b, 0, 0, -b])]


class PhaseDampingChannel(_SingleQubitChannel):
    """PhaseDampingChannel.java:51-63."""

    kind = "phase damping"

    def __init__(self, lam: float, qubits):
        _check_unit("lambda", lam)
        super().__init__(qubits)
        self.lam = lam

    def krausDecomposition(self):
        lam = self.lam
        return [KrausOperator([1, 0, 0, math.sqrt(1.0 - lam)]),
                KrausOperator([0, 0, 0, math.sqrt(lam)])]


class ThermalRelaxationChannel(_SingleQubitChannel):
    """ThermalRelaxationChannel.java (buildKrausDecomposition, boundedFactor, nonNegativeRate)."""

    kind = "thermal relaxation"
    _BOUNDED = 1e-12
    _RATE = 1e-12

    def __init__(self, t1: float, t2: float, gate_time: float, qubits):
        if t1 <= 0.0 or not math.isfinite(t1):
            raise ValueError(f"T1 must be positive and finite, got {t1}")
        if t2 <= 0.0 or not math.isfinite(t2):
            raise ValueError(f"T2 must be positive and finite, got {t2}")
        if t2 > 2.0 * t1:
            raise ValueError(f"T2 must satisfy T2 <= 2*T1 (physical constraint), got T1={t1}, T2={t2}")
        if gate_time < 0.0 or not math.isfinite(gate_time):
            raise ValueError(f"gate time must be non-negative and finite, got {gate_time}")
        super().__init__(qubits)
        self.t1, self.t2, self.gate_time = t1, t2, gate_time
        self._ops = self._build()

    @classmethod
    def _bounded(cls, name, v):
        if not math.isfinite(v):
            raise RuntimeError(f"{name} must be finite, got {v}")
        if v < 0.0:
            if v >= -cls._BOUNDED:
                return 0.0
            raise RuntimeError(f"{name} must be in [0,1], got {v}")
        if v > 1.0:
            if v <= 1.0 + cls._BOUNDED:
                return 1.0
            raise RuntimeError(f"{name} must be in [0,1], got {v}")
        return v

    @classmethod
    def _rate(cls, name, v, scale):
        if not math.isfinite(v):
            raise RuntimeError(f"{name} must be finite, got {v}")
        if v < 0.0:
            if v >= -cls._RATE * max(1.0, scale):
                return 0.0
            raise RuntimeError(f"{name} must be non-negative, got {v}")
        return v

    def _build(self):
        if self.gate_time == 0.0:
            surv, deph = 1.0, 1.0
        else:
            surv = self._bounded("relaxation survival", math.exp(-self.gate_time / self.t1))
            inv_t2 = 1.0 / self.t2
            half_inv_t1 = 1.0 / (2.0 * self.t1)
            rate = self._rate("pure dephasing rate", inv_t2 - half_inv_t1,
                              abs(inv_t2) + abs(half_inv_t1))
            deph = self._bounded("pure dephasing factor", math.exp(-self.gate_time * rate))
        decay = self._bounded("decay probability", 1.0 - surv)
        sqrt_surv = math.sqrt(surv)
        plus = self._bounded("thermal plus factor", 0.5 * (1.0 + deph))
        minus = self._bounded("thermal minus factor", 0.5 * (1.0 - deph))
        k0d0 = math.sqrt(plus)
        k0d1 = sqrt_surv * k0d0
        k1d0 = math.sqrt(minus)
        k1d1 = sqrt_surv * k1d0
        return [KrausOperator([k0d0, 0, 0, k0d1]),
                KrausOperator([k1d0, 0, 0, -k1d1]),
                KrausOperator([0, math.sqrt(decay), 0, 0])]

    def krausDecomposition(self):
        return self._ops


class CompositeChannel(ErrorChannel):
    """CompositeChannel.java: components applied in sequence."""

    def __init__(self, channels: Sequence[ErrorChannel]):
        if not channels:
            raise ValueError("composite channel requires at least one channel")
        self.channels = tuple(channels)
        self._qubits = tuple(sorted({q for c in self.channels for q in c.affectedQubits()}))

    def krausDecomposition(self):
        raise NotImplementedError(
            "CompositeChannel does not provide a single Kraus decomposition. "
            "Use getChannels() for sequential application.")

    def affectedQubits(self):
        return self._qubits

    def getChannels(self):
        return tuple(self.channels)


def _is_single_qubit_channel(channel: ErrorChannel) -> bool:
    if isinstance(channel, CompositeChannel):
        return all(_is_single_qubit_channel(c) for c in channel.channels)
    return channel.krausDecomposition()[0].numQubits == 1


def java_integer_hashmap_order(keys_in_insertion_order: Sequence[int]) -> list[int]:
    """Iteration order of a java.util.HashMap<Integer, ?> filled in the given order.

    Bucket = (h ^ (h >>> 16)) & (capacity - 1) with h = the int value; capacity starts
    at 16 and doubles whenever size exceeds 0.75 * capacity; within a bucket entries
    keep insertion order (resize splits preserve it).
    """
    keys = list(dict.fromkeys(keys_in_insertion_order))
    cap = 16
    while len(keys) > 0.75 * cap:
        cap *= 2

    def bucket(k: int) -> int:
        h = k & 0xFFFFFFFF
        h ^= h >> 16
        return h & (cap - 1)

    return [k for _, _, k in sorted((bucket(k), i, k) for i, k in enumerate(keys))]


@dataclass(frozen=True)
class ScheduledChannel:
    channel: ErrorChannel
    targetQubits: tuple


class NoiseModel:
    """NoiseModel.java: gate-type, idle (per-qubit) and global channels."""

    def __init__(self):
        self._gate: dict[type, list[ErrorChannel]] = {}
        self._qubit: dict[int, list[ErrorChannel]] = {}
        self._qubit_insertion: list[int] = []
        self._global: list[ErrorChannel] = []

    @staticmethod
    def builder() -> "NoiseModel.Builder":
        return NoiseModel.Builder()

    def afterGate(self, gate_type: type, channel: ErrorChannel) -> "NoiseModel":
        self._gate.setdefault(gate_type, []).append(channel)
        return self

    def onQubits(self, channel: ErrorChannel, *qubits: int) -> "NoiseModel":
        if not qubits:
            raise ValueError("must specify at least one qubit")
        seen = set()
        for q in qubits:
            if q < 0:
                raise ValueError("qubit index must be non-negative")
            if q in seen:
                raise ValueError(f"duplicate qubit index: {q}")
            seen.add(q)
        if not _is_single_qubit_channel(channel):
            raise ValueError("onQubits requires channels that decompose to single-qubit operators")
        for q in qubits:
            if q not in self._qubit:
                self._qubit[q] = []
                self._qubit_insertion.append(q)
            self._qubit[q].append(channel)
        return self

    def afterAllGates(self, channel: ErrorChannel) -> "NoiseModel":
        self._global.append(channel)
        return self

    def hasNoise(self) -> bool:
        return bool(self._gate or self._qubit or self._global)

    def scheduledChannelsAfter(self, operation: Q.Operation) -> list[ScheduledChannel]:
        out: list[ScheduledChannel] = []
        for ch in self._gate.get(type(operation), []):
            out.append(ScheduledChannel(ch, tuple(ch.affectedQubits())))
        touched = set(operation.qubits_touched())
        for q in java_integer_hashmap_order(self._qubit_insertion):
            if q in touched:
                continue
            for ch in self._qubit[q]:
                out.append(ScheduledChannel(ch, (q,)))
        for ch in self._global:
            out.append(ScheduledChannel(ch, tuple(ch.affectedQubits())))
        return out

    class Builder:
        def __init__(self):
            self._model = NoiseModel()

        def afterGate(self, gate_type: type, channel: ErrorChannel):
            self._model.afterGate(gate_type, channel)
            return self

        def onQubits(self, channel: ErrorChannel, *qubits: int):
            self._model.onQubits(channel, *qubits)
            return self

        def afterAllGates(self, channel: ErrorChannel):
            self._model.afterAllGates(channel)
            return self

        def build(self) -> "NoiseModel":
            built = NoiseModel()
            built._gate = {k: list(v) for k, v in self._model._gate.items()}
            order = java_integer_hashmap_order(self._model._qubit_insertion)
            built._qubit = {q: list(self._model._qubit[q]) for q in order}
            built._qubit_insertion = order
            built._global = list(self._model._global)
            return built


@dataclass(frozen=True)
class FlatChannel:
    """One (channel, target) application: the host form of ``sc_channel``."""

    after_op: int
    target: int
    kraus: tuple  # of 2x2 numpy arrays


def _resolve_targets(mapped, channel: ErrorChannel, qubit_count: int) -> tuple[int, ...]:
    targets = tuple(mapped) if mapped is not None else tuple(channel.affectedQubits())
    if not targets:
        raise ValueError("noise channel must target at least one qubit")
    seen = set()
    for t in targets:
        if t < 0 or t >= qubit_count:
            raise ValueError(f"noise channel qubit out of range: {t}")
        if t in seen:
            raise ValueError(f"noise channel contains duplicate qubit: {t}")
        seen.add(t)
    return targets


def _flatten_channel(out: list, op_index: int, channel: ErrorChannel, mapped, qubit_count: int):
    if isinstance(channel, CompositeChannel):
        component_mapping = mapped if mapped is not None and len(mapped) == 1 else None
        for comp in channel.channels:
            _flatten_channel(out, op_index, comp, component_mapping, qubit_count)
        return
    targets = _resolve_targets(mapped, channel, qubit_count)
    ops = channel.krausDecomposition()
    if ops[0].numQubits != 1:
        raise NotImplementedError("only single-qubit Kraus channels are supported")
    mats = tuple(np.array(k.matrix, dtype=np.complex128).reshape(2, 2) for k in ops)
    for t in targets:
        out.append(FlatChannel(op_index, t, mats))


def flatten_schedule(circuit: Q.QuantumCircuit, model: NoiseModel | None) -> list[FlatChannel]:
    """All channel applications of a noisy run, in the reference engine's order."""
    if model is None or not model.hasNoise():
        return []
    out: list[FlatChannel] = []
    for i, op in enumerate(circuit.operations):
        if isinstance(op, Q.MeasureOperation):
            continue
        for sched in model.scheduledChannelsAfter(op):
            _flatten_channel(out, i, sched.channel, sched.targetQubits, circuit.qubitCount)
    return out
