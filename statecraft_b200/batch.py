"""Batched QAOA ring ansatz on one B200 (``sc_qaoa_batch_*`` in the C ABI).

The reference runs a QAOA suite one circuit at a time through
``StatevectorEngine.simulate`` (the ansatz is ``AlgorithmSuiteSpecs.qaoaRingAnsatz``,
app/.../AlgorithmSuiteSpecs.java:186-200, cost phases :283-287).  Here a whole batch
of instances with uneven qubit counts runs as one captured CUDA graph and returns
``<sum_j Z_j Z_{j+1 mod n}>`` per instance, so a parameter sweep costs one graph
launch per step.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _abi as A
from .engine import B200Config, NativeContext

MAX_QUBITS = 23
MAX_LAYERS = 16


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class QaoaRingBatch:
    """Many QAOA ring-ansatz instances evaluated together.

    ``n_qubits[i]`` in 2..23; ``gammas`` / ``betas`` of shape (instances, p), p in 1..16.
    ``dtype`` is ``A.SC_C128`` or ``A.SC_C64`` (complex64 amplitudes, FP64 tables and
    reductions).  ``tune`` times the kernel shapes on this batch and keeps the fastest.
    """

    def __init__(self, n_qubits: Sequence[int], gammas, betas, dtype: int = A.SC_C128,
                 tune: bool = True, context: Optional[NativeContext] = None):
        self.n_qubits = np.ascontiguousarray(n_qubits, dtype=np.int32)
        g = np.ascontiguousarray(gammas, dtype=np.float64)
        b = np.ascontiguousarray(betas, dtype=np.float64)
        if g.ndim != 2 or g.shape != b.shape or g.shape[0] != self.n_qubits.size:
            raise ValueError("gammas and betas must both have shape (instances, layers)")
        self.p = int(g.shape[1])
        self.dtype = dtype
        self._own = context is None
        self.ctx = context or NativeContext(B200Config())
        self.lib = self.ctx.lib
        handle = ctypes.c_void_p()
        rc = self.lib.sc_qaoa_batch_create(
            self.ctx.handle, dtype, int(self.n_qubits.size),
            self.n_qubits.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), self.p,
            _dptr(g), _dptr(b), 1 if tune else 0, ctypes.byref(handle))
        A.raise_for(rc, self.lib)
        self.handle = handle

    @property
    def instances(self) -> int:
        return int(self.n_qubits.size)

    def set_angles(self, gammas, betas) -> None:
        g = np.ascontiguousarray(gammas, dtype=np.float64)
        b = np.ascontiguousarray(betas, dtype=np.float64)
        if g.shape != (self.instances, self.p) or b.shape != g.shape:
            raise ValueError("angle arrays must keep the batch's shape")
        A.raise_for(self.lib.sc_qaoa_batch_set_angles(self.handle, _dptr(g), _dptr(b)), self.lib)

    def run(self) -> None:
        """Enqueue one evaluation of the whole batch (asynchronous)."""
        A.raise_for(self.lib.sc_qaoa_batch_run(self.handle), self.lib)

    def energies(self, with_norms: bool = False):
        e = np.empty(self.instances)
        nrm = np.empty(self.instances)
        A.raise_for(self.lib.sc_qaoa_batch_energies(self.handle, _dptr(e), _dptr(nrm)), self.lib)
        return (e, nrm) if with_norms else e

    def evaluate(self):
        self.run()
        return self.energies()

    def info(self) -> dict:
        nr = ctypes.c_int32()
        ctas = ctypes.c_int32()
        ms = ctypes.c_double()
        by = ctypes.c_double()
        A.raise_for(self.lib.sc_qaoa_batch_info(self.handle, ctypes.byref(nr), ctypes.byref(ctas),
                                                ctypes.byref(ms), ctypes.byref(by)), self.lib)
        return {"register_qubits": nr.value, "ctas_per_sm": ctas.value,
                "tuned_ms": ms.value, "hbm_bytes_per_run": by.value}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.sc_qaoa_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()
        if getattr(self, "_own", False) and self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):  # pragma: no cover - interpreter teardown
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def amp_updates(n_qubits: Sequence[int], p: int) -> float:
        """Gate-level amplitude updates of one batch evaluation: per instance n H gates,
        and per layer n ring ZZ phases and n RX, each touching 2^n amplitudes."""
        n = np.asarray(n_qubits, dtype=np.float64)
        return float(np.sum((n + 2.0 * p * n) * np.exp2(n)))
