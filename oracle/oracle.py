"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper around ``oracle/_build/libsc_oracle.so`` (built from
``oracle/sc_oracle.c`` by ``make -C oracle``), the plain-C restatement of the
reference ``statevector`` engine (StatevectorOps.java, StatevectorEngine.java,
ComplexArrays.java, SplittableRandom).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, and only as the checker; the product package
never imports it.

``simulate_request`` mirrors StatevectorEngine.simulate (StatevectorEngine.java:63-167)
end to end on the CPU, reusing the product's host-side request serialisation so
both sides consume identical sc_op / sc_channel records.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB = ORACLE_DIR / "_build" / "libsc_oracle.so"

_lib = None

_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_ip = _P(ctypes.c_int32)


class ScxRng(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("gamma", ctypes.c_uint64)]


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    from statecraft_b200 import _abi as A  # struct layouts only

    lib = ctypes.CDLL(str(LIB))
    sig = {
        "scx_rng_seed": (None, [_P(ScxRng), ctypes.c_uint64]),
        "scx_rng_next_long": (ctypes.c_uint64, [_P(ScxRng)]),
        "scx_rng_next_double": (ctypes.c_double, [_P(ScxRng)]),
        "scx_rng_next_double_bound": (ctypes.c_double, [_P(ScxRng), ctypes.c_double]),
        "scx_uniforms": (None, [ctypes.c_uint64, ctypes.c_int64, _dp]),
        "scx_apply_op": (ctypes.c_int, [_dp, ctypes.c_int, _P(A.ScOp), _dp, ctypes.c_int64]),
        "scx_run": (ctypes.c_int, [_dp, ctypes.c_int, _P(A.ScOp), ctypes.c_int64, _dp,
                                   ctypes.c_int64, _P(A.ScChannel), ctypes.c_int64,
                                   ctypes.c_uint64, _ip]),
        "scx_norm2sq": (ctypes.c_double, [_dp, ctypes.c_int64]),
        "scx_probabilities": (None, [_dp, ctypes.c_int, _ip, ctypes.c_int, _dp]),
        "scx_normalize": (ctypes.c_int, [_dp, ctypes.c_int64]),
        "scx_cumulative": (None, [_dp, ctypes.c_int64, _dp]),
        "scx_sample_outcome": (ctypes.c_int64, [_dp, ctypes.c_int64, ctypes.c_double]),
        "scx_sample": (ctypes.c_int, [_dp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int64,
                                      ctypes.c_uint64, _dp, _ip]),
        "scx_expect_pauli": (ctypes.c_double, [_dp, ctypes.c_int, ctypes.c_int32,
                                               _P(ctypes.c_uint64), _P(ctypes.c_uint64), _dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class SplittableRandom:
    """The oracle's SplitMix64 (java.util.SplittableRandom restatement)."""

    def __init__(self, seed: int):
        self._r = ScxRng()
        load().scx_rng_seed(ctypes.byref(self._r), seed & 0xFFFFFFFFFFFFFFFF)

    def nextLong(self) -> int:
        return load().scx_rng_next_long(ctypes.byref(self._r))

    def nextDouble(self, bound: float | None = None) -> float:
        if bound is None:
            return load().scx_rng_next_double(ctypes.byref(self._r))
        return load().scx_rng_next_double_bound(ctypes.byref(self._r), bound)


def uniforms(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    load().scx_uniforms(seed & 0xFFFFFFFFFFFFFFFF, count, _d(out))
    return out


def initial_state(n: int, init=None, basis_mask: int | None = None) -> np.ndarray:
    st = np.zeros(2 << n, dtype=np.float64)
    if init is not None:
        st[:] = np.asarray(init, dtype=np.float64).reshape(-1)
    else:
        st[2 * (basis_mask or 0)] = 1.0
    return st


def run(n: int, ops, n_ops: int, state: np.ndarray, channels=None, n_channels: int = 0,
        noise_seed: int = 0, params: np.ndarray | None = None):
    """Runs ops in place on `state`; returns (status, chosen Kraus indices)."""
    lib = load()
    chosen = np.full(max(1, n_channels), -1, dtype=np.int32)
    p = None
    n_params = 0
    if params is not None:
        params = np.ascontiguousarray(params, dtype=np.float64)
        p = _d(params)
        n_params = params.size
    rc = lib.scx_run(_d(state), n, ops, n_ops, p, n_params, channels, n_channels,
                     noise_seed & 0xFFFFFFFFFFFFFFFF, _i(chosen))
    return rc, chosen[:n_channels]


def norm2sq(state: np.ndarray) -> float:
    return load().scx_norm2sq(_d(state), state.size // 2)


def probabilities(state: np.ndarray, n: int, qubits) -> np.ndarray:
    q = np.ascontiguousarray(qubits, dtype=np.int32)
    out = np.empty(1 << q.size, dtype=np.float64)
    load().scx_probabilities(_d(state), n, _i(q), q.size, _d(out))
    return out


def cumulative(probs: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(probs, dtype=np.float64).copy()
    rc = load().scx_normalize(_d(p), p.size)
    if rc != 0:
        raise RuntimeError("State collapsed to zero probability amplitudes")
    cdf = np.empty_like(p)
    load().scx_cumulative(_d(p), p.size, _d(cdf))
    return cdf


def sample_outcome(cdf: np.ndarray, u: float) -> int:
    return load().scx_sample_outcome(_d(cdf), cdf.size, u)


def sample(state: np.ndarray, n: int, qubits, shots: int, seed: int,
           uniforms_: np.ndarray | None = None) -> np.ndarray:
    q = np.ascontiguousarray(qubits, dtype=np.int32)
    out = np.empty(shots, dtype=np.int32)
    u = None
    if uniforms_ is not None:
        uniforms_ = np.ascontiguousarray(uniforms_, dtype=np.float64)
        u = _d(uniforms_)
    rc = load().scx_sample(_d(state), n, _i(q), q.size, shots, seed & 0xFFFFFFFFFFFFFFFF, u,
                           _i(out))
    if rc != 0:
        raise RuntimeError(f"oracle sampling failed: {rc}")
    return out


def expect_pauli(state: np.ndarray, n: int, xmask, zmask, coeffs) -> float:
    x = np.ascontiguousarray(xmask, dtype=np.uint64)
    z = np.ascontiguousarray(zmask, dtype=np.uint64)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    u64 = _P(ctypes.c_uint64)
    return load().scx_expect_pauli(_d(state), n, c.size, x.ctypes.data_as(u64),
                                   z.ctypes.data_as(u64), _d(c))


def simulate_request(request):
    """StatevectorEngine.simulate restated on the oracle.

    Returns (final interleaved state, measurement dict or None, chosen Kraus indices).
    Raises the same exception types as the engine.
    """
    from statecraft_b200 import _abi as A
    from statecraft_b200 import engine as E
    from statecraft_b200 import noise as N
    from statecraft_b200 import quantum as Q

    circuit = request.circuit
    n = circuit.qubitCount
    ops, n_ops = E.serialize_circuit(circuit)
    flat = N.flatten_schedule(circuit, request.noiseModel) if request.noiseModel else []
    ch, n_ch = E.serialize_channels(flat)
    basis = None
    init = None
    if request.initialState is not None:
        init = request.initialState.copyData()
    elif request.basisStateQubits is not None:
        basis = sum(1 << q for q in request.basisStateQubits)
    st = initial_state(n, init, basis)
    seed = request.noiseSeed if request.noiseSeed is not None else 0
    rc, chosen = run(n, ops, n_ops, st, ch, n_ch, seed)
    if rc == A.SC_EUNSUPPORTED:
        raise A.UnsupportedOperationException("Unitary operations cannot follow measurement "
                                              "operations in the circuit")
    if rc == A.SC_EINVAL:
        raise A.IllegalArgumentException("invalid operation or noise target")
    if rc == A.SC_ESTATE:
        raise A.IllegalStateException("invalid Kraus branch weights / norm")
    measurement = None
    instr = request.measurement
    if instr is not None:
        qubits = instr.measuredQubits
        if qubits is None:
            measured = sorted({q for op in circuit.operations
                               if isinstance(op, Q.MeasureOperation) for q in op.qubits})
            qubits = tuple(measured) if measured else tuple(range(n))
        outcomes = sample(st, n, qubits, instr.shots, instr.seed if instr.seed is not None else 0)
        measurement = {"qubits": tuple(qubits), "outcomes": outcomes}
    return st, measurement, chosen


def qaoa_ring_energy(n: int, gammas, betas) -> float:
    """<sum_j Z_j Z_{j+1 mod n}> of the QAOA ring ansatz (H on all qubits, then per layer
    the ring ZZ phases and RX(2 beta), AlgorithmSuiteSpecs.java:186-200), gate by gate
    on the oracle."""
    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import serialize_circuit

    c = W.qaoa_circuit(n, gammas, betas)
    ops, n_ops = serialize_circuit(c)
    st = initial_state(n)
    rc, _ = run(n, ops, n_ops, st)
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    z = [(1 << j) | (1 << ((j + 1) % n)) for j in range(n)]
    return expect_pauli(st, n, [0] * n, z, [1.0] * n)
