"""Engine SPI mirror and the B200 statevector engine.

Mirrors core/.../core/engine/ (SimulatorEngine.java, SimulatorEngines.java,
SimulationRequest.java, MeasurementInstruction.java, MeasurementResult.java,
SimulationResult.java) and implements ``StatevectorB200Engine``, the drop-in for
engines/.../statevector/StatevectorEngine.java registered under the id
``statevector-b200``.  The engine only flattens the request and calls the C ABI;
every amplitude is computed on the GPU.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass, field
from enum import Enum
from typing import Optional, Sequence

import numpy as np

from . import _abi as A
from . import noise as N
from . import quantum as Q

# --------------------------------------------------------------------------
# requests / results
# --------------------------------------------------------------------------


class Mode(Enum):
    COUNTS = "COUNTS"
    SAMPLES = "SAMPLES"


def _normalize_qubits(qubits: Sequence[int]) -> tuple[int, ...]:
    if len(qubits) == 0:
        raise ValueError("measured qubit list must not be empty")
    for q in qubits:
        if q < 0:
            raise ValueError(f"qubit index must be non-negative: {q}")
    qs = tuple(sorted(int(q) for q in qubits))
    for a, b in zip(qs, qs[1:]):
        if a == b:
            raise ValueError(f"duplicate qubit index: {b}")
    return qs


@dataclass(frozen=True)
class MeasurementInstruction:
    """MeasurementInstruction.java:12-85."""

    shots: int
    measuredQubits: Optional[tuple] = None
    seed: Optional[int] = None
    mode: Mode = Mode.COUNTS

    def __post_init__(self):
        if self.shots <= 0:
            raise ValueError("shots must be positive")
        if self.measuredQubits is not None:
            object.__setattr__(self, "measuredQubits", _normalize_qubits(self.measuredQubits))

    def withSeed(self, seed: int) -> "MeasurementInstruction":
        return MeasurementInstruction(self.shots, self.measuredQubits, int(seed), self.mode)

    def withoutSeed(self) -> "MeasurementInstruction":
        return MeasurementInstruction(self.shots, self.measuredQubits, None, self.mode)

    @staticmethod
    def countsAll(shots: int) -> "MeasurementInstruction":
        return MeasurementInstruction(shots, None, None, Mode.COUNTS)

    @staticmethod
    def counts(shots: int, *qubits: int) -> "MeasurementInstruction":
        if not qubits:
            raise ValueError("at least one qubit must be provided")
        return MeasurementInstruction(shots, tuple(qubits), None, Mode.COUNTS)

    @staticmethod
    def samplesAll(shots: int) -> "MeasurementInstruction":
        return MeasurementInstruction(shots, None, None, Mode.SAMPLES)

    @staticmethod
    def samples(shots: int, *qubits: int) -> "MeasurementInstruction":
        if not qubits:
            raise ValueError("at least one qubit must be provided")
        return MeasurementInstruction(shots, tuple(qubits), None, Mode.SAMPLES)


@dataclass(frozen=True)
class SimulationRequest:
    """SimulationRequest.java:17-131 (same validation and builder methods)."""

    circuit: Q.QuantumCircuit
    initialState: Optional[Q.StateVector] = None
    basisStateQubits: Optional[tuple] = None
    measurement: Optional[MeasurementInstruction] = None
    noiseModel: Optional[N.NoiseModel] = None
    noiseSeed: Optional[int] = None
    returnFinalState: bool = True

    def __post_init__(self):
        if self.circuit is None:
            raise TypeError("circuit")
        n = self.circuit.qubitCount
        if self.initialState is not None and self.initialState.qubitCount() != n:
            raise ValueError(f"Initial state qubit count {self.initialState.qubitCount()} "
                             f"does not match circuit qubit count {n}")
        if self.basisStateQubits is not None:
            qs = sorted(int(q) for q in self.basisStateQubits)
            for q in qs:
                if q < 0 or q >= n:
                    raise ValueError(f"basis-state qubit out of range: {q}")
            for a, b in zip(qs, qs[1:]):
                if a == b:
                    raise ValueError(f"duplicate basis-state qubit: {b}")
            object.__setattr__(self, "basisStateQubits", tuple(qs))
        if self.initialState is not None and self.basisStateQubits is not None:
            raise ValueError("initialState and basisStateQubits are mutually exclusive")
        if self.measurement is not None and self.measurement.measuredQubits is not None:
            for q in self.measurement.measuredQubits:
                if q < 0 or q >= n:
                    raise ValueError(f"measurement qubit out of range: {q}")
        if not self.returnFinalState and self.measurement is None:
            raise ValueError(
                "simulation must request the final state or provide a measurement instruction")

    @staticmethod
    def zeroState(circuit: Q.QuantumCircuit) -> "SimulationRequest":
        return SimulationRequest(circuit)

    @staticmethod
    def withInitialState(circuit: Q.QuantumCircuit, state: Q.StateVector) -> "SimulationRequest":
        if state is None:
            raise TypeError("state")
        return SimulationRequest(circuit, initialState=state)

    def _replace(self, **kw) -> "SimulationRequest":
        fields = dict(circuit=self.circuit, initialState=self.initialState,
                      basisStateQubits=self.basisStateQubits, measurement=self.measurement,
                      noiseModel=self.noiseModel, noiseSeed=self.noiseSeed,
                      returnFinalState=self.returnFinalState)
        fields.update(kw)
        return SimulationRequest(**fields)

    def withMeasurement(self, instruction: MeasurementInstruction,
                        includeFinalState: Optional[bool] = None) -> "SimulationRequest":
        if instruction is None:
            raise TypeError("instruction")
        keep = self.returnFinalState if includeFinalState is None else includeFinalState
        return self._replace(measurement=instruction, returnFinalState=keep)

    def withoutFinalState(self) -> "SimulationRequest":
        if self.measurement is None:
            raise RuntimeError("cannot drop final state without measurement instruction")
        return self._replace(returnFinalState=False)

    def withNoiseModel(self, model: N.NoiseModel) -> "SimulationRequest":
        if model is None:
            raise TypeError("model")
        return self._replace(noiseModel=model)

    def withNoiseSeed(self, seed: int) -> "SimulationRequest":
        return self._replace(noiseSeed=int(seed))

    def withBasisState(self, *qubits: int) -> "SimulationRequest":
        return self._replace(initialState=None, basisStateQubits=tuple(qubits))


class MeasurementResult:
    pass


@dataclass(frozen=True)
class Histogram(MeasurementResult):
    """MeasurementResult.Histogram: outcome bit k <-> measuredQubits[k]."""

    measuredQubits: tuple
    shots: int
    counts: dict


@dataclass(frozen=True)
class Samples(MeasurementResult):
    measuredQubits: tuple
    shots: int
    outcomes: tuple


@dataclass(frozen=True)
class SimulationResult:
    finalState: Optional[Q.StateVector] = None
    measurement: Optional[MeasurementResult] = None


class SimulatorEngine:
    """SimulatorEngine.java:5-8."""

    def id(self) -> str:  # pragma: no cover - abstract
        raise NotImplementedError

    def simulate(self, request: SimulationRequest) -> SimulationResult:  # pragma: no cover
        raise NotImplementedError


# --------------------------------------------------------------------------
# op-stream serialisation
# --------------------------------------------------------------------------


def _put_complex(dst, values: Sequence[complex]) -> None:
    for k, v in enumerate(values):
        dst[2 * k] = v.real
        dst[2 * k + 1] = v.imag


def _gate_entries(gate: Q.SingleQubitGate) -> list[complex]:
    return [gate.element(0, 0), gate.element(0, 1), gate.element(1, 0), gate.element(1, 1)]


def serialize_circuit(circuit: Q.QuantumCircuit):
    """QuantumCircuit.operations() -> ctypes array of sc_op."""
    ops = circuit.operations
    arr = (A.ScOp * max(1, len(ops)))()
    for i, op in enumerate(ops):
        rec = arr[i]
        rec.q1 = -1
        rec.param = -1
        if isinstance(op, Q.SingleGateOperation):
            rec.kind = A.SC_OP_SINGLE
            rec.q0 = op.qubit
            _put_complex(rec.m, _gate_entries(op.gate))
        elif isinstance(op, Q.CnotOperation):
            rec.kind = A.SC_OP_CNOT
            rec.q0, rec.q1 = op.controlQubit, op.targetQubit
        elif isinstance(op, Q.TwoQubitGateOperation):
            rec.kind = A.SC_OP_TWO
            rec.q0, rec.q1 = op.firstQubit, op.secondQubit
            _put_complex(rec.m, op.matrix)
        elif isinstance(op, Q.TwoQubitDiagonalOperation):
            rec.kind = A.SC_OP_DIAG2
            rec.q0, rec.q1 = op.firstQubit, op.secondQubit
            _put_complex(rec.m, op.diagonal)
        elif isinstance(op, Q.SwapOperation):
            rec.kind = A.SC_OP_SWAP
            rec.q0, rec.q1 = op.firstQubit, op.secondQubit
        elif isinstance(op, Q.MultiControlOperation):
            rec.kind = A.SC_OP_MULTI
            rec.q0 = op.targetQubit
            mask = 0
            for c in op.controlQubits:
                mask |= 1 << c
            rec.mask = mask
            _put_complex(rec.m, _gate_entries(op.gate))
        elif isinstance(op, Q.MeasureOperation):
            rec.kind = A.SC_OP_MEASURE
            mask = 0
            for q in op.qubits:
                mask |= 1 << q
            rec.mask = mask
        else:
            raise RuntimeError(f"Unsupported operation type: {type(op).__name__}")
    return arr, len(ops)


def serialize_channels(flat: Sequence[N.FlatChannel]):
    arr = (A.ScChannel * max(1, len(flat)))()
    for i, fc in enumerate(flat):
        rec = arr[i]
        rec.after_op = fc.after_op
        rec.target = fc.target
        if len(fc.kraus) > A.SC_MAX_KRAUS:
            raise NotImplementedError(f"at most {A.SC_MAX_KRAUS} Kraus operators per channel")
        rec.n_kraus = len(fc.kraus)
        for k, mat in enumerate(fc.kraus):
            _put_complex(rec.kraus[k], list(mat.reshape(-1)))
    return arr, len(flat)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


# --------------------------------------------------------------------------
# native context wrapper
# --------------------------------------------------------------------------


@dataclass
class B200Config:
    """Engine configuration (device ordinal, amplitude type, fusion settings)."""

    device: int = 0
    dtype: int = A.SC_C128
    fusion: bool = True
    tile_qubits: int = 0
    sweep_budget: int = 0
    max_qubits: int = 0
    timing: bool = False
    device_mem_limit: int = 0
    autotune: bool = False

    def to_native(self) -> A.ScConfig:
        cfg = A.ScConfig()
        cfg.dtype = self.dtype
        cfg.fusion = 1 if self.fusion else 0
        cfg.tile_qubits = self.tile_qubits
        cfg.sweep_budget = self.sweep_budget
        cfg.max_qubits = self.max_qubits
        cfg.timing = 1 if self.timing else 0
        cfg.device_mem_limit = self.device_mem_limit
        cfg.autotune = 1 if self.autotune else 0
        return cfg


class NativeContext:
    """Owns one ``sc_ctx`` (device state buffer + stream)."""

    def __init__(self, config: B200Config | None = None):
        self.lib = A.load()
        self.config = config or B200Config()
        handle = ctypes.c_void_p()
        cfg = self.config.to_native()
        A.raise_for(self.lib.sc_create(self.config.device, ctypes.byref(cfg),
                                       ctypes.byref(handle)), self.lib)
        self.handle = handle

    def close(self) -> None:
        if self.handle:
            self.lib.sc_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter teardown
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> int:
        A.raise_for(rc, self.lib)
        return rc

    def set_noise(self, flat: Sequence[N.FlatChannel], seed: Optional[int]) -> None:
        arr, n = serialize_channels(flat)
        s = 0 if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF
        self._check(self.lib.sc_set_noise(self.handle, arr, n, s, 0 if seed is None else 1))

    def run_ops(self, n_qubits: int, ops, n_ops: int, init: Optional[np.ndarray] = None,
                basis_mask: Optional[int] = None) -> None:
        init_ptr = None
        if init is not None:
            init = np.ascontiguousarray(init, dtype=np.float64)
            if init.size != 2 << n_qubits:
                raise ValueError("initial state length mismatch")
            init_ptr = _dptr(init)
        self._check(self.lib.sc_run(self.handle, n_qubits, ops, n_ops, init_ptr,
                                    0 if basis_mask is None else basis_mask,
                                    0 if basis_mask is None else 1))

    def state(self, n_qubits: int) -> np.ndarray:
        out = np.empty(2 << n_qubits, dtype=np.float64)
        self._check(self.lib.sc_get_state(self.handle, _dptr(out), out.size))
        return out

    def default_measured_qubits(self, cap: int = 64) -> tuple[int, ...]:
        buf = np.empty(cap, dtype=np.int32)
        count = self._check(self.lib.sc_default_measured_qubits(self.handle, _iptr(buf), cap))
        return tuple(int(x) for x in buf[:count])

    def sample(self, qubits: Sequence[int], shots: int, seed: Optional[int],
               uniforms: Optional[np.ndarray] = None) -> np.ndarray:
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        out = np.empty(shots, dtype=np.int32)
        u_ptr = None
        if uniforms is not None:
            uniforms = np.ascontiguousarray(uniforms, dtype=np.float64)
            if uniforms.size < shots:
                raise ValueError("need one uniform per shot")
            u_ptr = _dptr(uniforms)
        s = 0 if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF
        self._check(self.lib.sc_sample(self.handle, _iptr(q), q.size, shots, s,
                                       0 if seed is None else 1, u_ptr, _iptr(out)))
        return out

    def probabilities(self, qubits: Sequence[int]) -> np.ndarray:
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        out = np.empty(1 << q.size, dtype=np.float64)
        self._check(self.lib.sc_probabilities(self.handle, _iptr(q), q.size, _dptr(out)))
        return out

    def expect_pauli(self, xmask: Sequence[int], zmask: Sequence[int],
                     coeffs: Sequence[float]) -> float:
        x = np.ascontiguousarray(xmask, dtype=np.uint64)
        z = np.ascontiguousarray(zmask, dtype=np.uint64)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        out = ctypes.c_double()
        u64p = ctypes.POINTER(ctypes.c_uint64)
        self._check(self.lib.sc_expect_pauli(self.handle, c.size, x.ctypes.data_as(u64p),
                                             z.ctypes.data_as(u64p), _dptr(c),
                                             ctypes.byref(out)))
        return out.value

    def kernel_stats(self) -> dict:
        cap = 32
        launches = np.zeros(cap, dtype=np.int64)
        ms = np.zeros(cap, dtype=np.float64)
        nbytes = np.zeros(cap, dtype=np.float64)
        count = self._check(self.lib.sc_kernel_stats(
            self.handle, launches.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dptr(ms),
            _dptr(nbytes), cap))
        out = {}
        for i in range(count):
            name = self.lib.sc_kernel_class_name(i).decode()
            out[name] = {"launches": int(launches[i]), "ms": float(ms[i]),
                         "bytes": float(nbytes[i])}
        return out

    def reset_kernel_stats(self) -> None:
        self._check(self.lib.sc_reset_kernel_stats(self.handle))

    def trajectories_info(self) -> dict:
        """Shape, graph and tuning time of the context's last trajectory batch."""
        t, r, g = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        ms = ctypes.c_double()
        self._check(self.lib.sc_trajectories_info(self.handle, ctypes.byref(t), ctypes.byref(r),
                                                  ctypes.byref(g), ctypes.byref(ms)))
        return {"tile_qubits": t.value, "nr": r.value, "graph": g.value, "tuned_ms": ms.value}

    def plan_stats(self) -> dict:
        s, g, st = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.sc_last_plan_stats(self.handle, ctypes.byref(s), ctypes.byref(g),
                                                ctypes.byref(st)))
        return {"sweeps": s.value, "gates": g.value, "stages": st.value}


# --------------------------------------------------------------------------
# the engine
# --------------------------------------------------------------------------


class StatevectorB200Engine(SimulatorEngine):
    """Drop-in for StatevectorEngine (StatevectorEngine.java:32-167) on one B200."""

    ID = "statevector-b200"

    def __init__(self, config: B200Config | None = None):
        self.config = config or B200Config()
        self._ctx: Optional[NativeContext] = None
        self._lock = threading.Lock()
        self.last_qubit_count = 0

    def id(self) -> str:
        return self.ID

    def context(self) -> NativeContext:
        if self._ctx is None:
            self._ctx = NativeContext(self.config)
        return self._ctx

    def close(self) -> None:
        if self._ctx is not None:
            self._ctx.close()
            self._ctx = None

    def simulate(self, request: SimulationRequest) -> SimulationResult:
        if request is None:
            raise TypeError("request")
        circuit = request.circuit
        n = circuit.qubitCount
        ops, n_ops = serialize_circuit(circuit)
        model = request.noiseModel
        flat = N.flatten_schedule(circuit, model) if model is not None else []
        init = None
        basis = None
        if request.initialState is not None:
            init = request.initialState.copyData()
        elif request.basisStateQubits is not None:
            basis = 0
            for q in request.basisStateQubits:
                basis |= 1 << q
        with self._lock:
            ctx = self.context()
            ctx.set_noise(flat, request.noiseSeed if (model and model.hasNoise()) else None)
            ctx.run_ops(n, ops, n_ops, init, basis)
            self.last_qubit_count = n
            final_state = None
            if request.returnFinalState:
                if n > Q.StateVector.MAX_DENSE_QUBITS:
                    raise A.UnsupportedOperationException(
                        f"final state of {n} qubits exceeds the dense StateVector limit "
                        f"({Q.StateVector.MAX_DENSE_QUBITS}); use final_state_array()")
                final_state = Q.StateVector(n, ctx.state(n))
            measurement = None
            if request.measurement is not None:
                measurement = self._measure(ctx, n, request.measurement)
        return SimulationResult(final_state, measurement)

    def final_state_array(self) -> np.ndarray:
        """Side channel for states beyond the Java array limit (interleaved doubles)."""
        with self._lock:
            return self.context().state(self.last_qubit_count)

    def _measure(self, ctx: NativeContext, n: int, instr: MeasurementInstruction):
        qubits = instr.measuredQubits
        if qubits is None:
            qubits = ctx.default_measured_qubits(max(64, n))
        if len(qubits) == 0:
            raise A.IllegalStateException("No qubits available for measurement")
        outcomes = ctx.sample(qubits, instr.shots, instr.seed)
        if instr.mode == Mode.COUNTS:
            values, counts = np.unique(outcomes, return_counts=True)
            hist = {int(v): int(c) for v, c in zip(values, counts)}
            return Histogram(tuple(qubits), instr.shots, hist)
        return Samples(tuple(qubits), instr.shots, tuple(int(x) for x in outcomes))


class SimulatorEngines:
    """ServiceLoader-style registry (SimulatorEngines.java:23-51), B200 engines only."""

    _factories = {StatevectorB200Engine.ID: StatevectorB200Engine}

    @classmethod
    def loadAll(cls) -> list[SimulatorEngine]:
        return [cls._factories[k]() for k in sorted(cls._factories)]

    @classmethod
    def ids(cls) -> list[str]:
        return sorted(cls._factories)

    @classmethod
    def findById(cls, engine_id: str) -> Optional[SimulatorEngine]:
        factory = cls._factories.get(engine_id)
        return factory() if factory else None

    @classmethod
    def require(cls, engine_id: str) -> SimulatorEngine:
        engine = cls.findById(engine_id)
        if engine is None:
            raise ValueError(f"Unknown simulator engine: {engine_id}")
        return engine
