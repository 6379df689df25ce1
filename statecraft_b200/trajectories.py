"""Batched noisy trajectories on one B200 (``sc_trajectories`` in the C ABI).

The reference engine samples one Monte-Carlo trajectory per ``simulate`` call
(StatevectorEngine.java:371-600); a study over many trajectories runs the call in a
loop, trajectory t with noise seed S + t (StatecraftComparisonRunner.java:75).  Here
all trajectories of a circuit run as one batch: each trajectory draws its branches
from the same SplittableRandom stream the reference would use, and each sweep of the
fused plan is one kernel launch over every trajectory's state.  Pauli-mixture
records (depolarizing, phase flip) are drawn on the host and applied inside the
sweeps; records with state-dependent weights (amplitude / phase damping, thermal
relaxation) split the plan and are weighed, drawn and applied on the device for all
trajectories at once.  A repeated call with the same circuit and records replays a
captured CUDA graph (``NativeContext.trajectories_info``); ``B200Config(autotune=True)``
times a few tile shapes on the first batch and keeps the fastest.
"""
from __future__ import annotations

import collections
import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _abi as A
from . import noise as N
from . import quantum as Q
from .engine import B200Config, NativeContext, serialize_channels, serialize_circuit


def touched_qubit_depolarizing(circuit: Q.QuantumCircuit, p: float) -> list[N.FlatChannel]:
    """A single-qubit depolarizing channel after every gate on every qubit it touches
    (control and target of a CNOT), in gate order; NoiseModel has no such schedule
    (its gate channels name fixed qubits), so it is built directly as records."""
    kraus = tuple(np.array(k.matrix, dtype=complex).reshape(2, 2)
                  for k in N.DepolarizingChannel(p, (0,)).krausDecomposition())
    out = []
    for i, op in enumerate(circuit.operations):
        if isinstance(op, Q.MeasureOperation):
            continue
        for q in sorted(op.qubits_touched()):
            out.append(N.FlatChannel(i, q, kraus))
    return out


@dataclass
class TrajectoryResult:
    outcomes: np.ndarray                 # (trajectories, shots) basis indices
    choices: np.ndarray                  # (trajectories, records) chosen Kraus index
    states: Optional[np.ndarray] = None  # (trajectories, 2^n) complex, when requested

    def histogram(self) -> dict:
        """Outcome counts aggregated over all trajectories."""
        return dict(collections.Counter(self.outcomes.reshape(-1).tolist()))


def run_trajectories(circuit: Q.QuantumCircuit, records: Sequence[N.FlatChannel],
                     trajectories: int, noise_seed: int, shots: int, measure_seed: int,
                     return_states: bool = False,
                     context: Optional[NativeContext] = None) -> TrajectoryResult:
    """Runs ``trajectories`` trajectories of ``circuit`` with the noise ``records``.
    Trajectory t uses noise seed ``noise_seed + t`` and measurement seed
    ``measure_seed + t``."""
    own = context is None
    ctx = context or NativeContext(B200Config())
    try:
        n = circuit.qubitCount
        ops, n_ops = serialize_circuit(circuit)
        ch, n_ch = serialize_channels(records)
        outcomes = np.zeros((trajectories, max(shots, 0)), dtype=np.int32)
        choices = np.zeros((trajectories, max(n_ch, 1)), dtype=np.int32)
        states = np.zeros(trajectories * (2 << n)) if return_states else None
        ip = ctypes.POINTER(ctypes.c_int32)
        rc = ctx.lib.sc_trajectories(
            ctx.handle, n, ops, n_ops, ch, n_ch, trajectories,
            int(noise_seed) & 0xFFFFFFFFFFFFFFFF, shots, int(measure_seed) & 0xFFFFFFFFFFFFFFFF,
            outcomes.ctypes.data_as(ip) if shots > 0 else None, choices.ctypes.data_as(ip),
            states.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if return_states else None)
        A.raise_for(rc, ctx.lib)
        st = None
        if return_states:
            st = (states[0::2] + 1j * states[1::2]).reshape(trajectories, 1 << n)
        return TrajectoryResult(outcomes, choices[:, :n_ch], st)
    finally:
        if own:
            ctx.close()


def total_variation(a: dict, b: dict) -> float:
    """Total-variation distance between two outcome histograms."""
    na = sum(a.values())
    nb = sum(b.values())
    keys = set(a) | set(b)
    return 0.5 * sum(abs(a.get(k, 0) / na - b.get(k, 0) / nb) for k in keys)
