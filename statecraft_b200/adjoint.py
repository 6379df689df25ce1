"""Adjoint-differentiation forward/backward pair (addition; no counterpart in the
reference engine).  <H> = sum_k c_k <psi(theta)|P_k|psi(theta)> and its gradient
over every rotation angle in one reverse sweep on the GPU
(Jones & Gacon, arXiv:2009.02823).

Circuits are sc_op arrays whose SC_OP_RX/RY/RZ/RZZ records reference a parameter
index; other op kinds are fixed gates.  Hamiltonian terms are (xmask, zmask, coeff):
X on xmask bits, Z on zmask bits, Y where both are set.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi as A
from .engine import B200Config, NativeContext

_u64p = ctypes.POINTER(ctypes.c_uint64)
_dp = ctypes.POINTER(ctypes.c_double)


class AdjointEngine:
    def __init__(self, config: B200Config | None = None):
        self.ctx = NativeContext(config or B200Config())
        self._n_params = 0

    def close(self) -> None:
        self.ctx.close()

    def forward(self, n_qubits: int, ops, n_ops: int, params, xmask, zmask, coeffs) -> float:
        p = np.ascontiguousarray(params, dtype=np.float64)
        x = np.ascontiguousarray(xmask, dtype=np.uint64)
        z = np.ascontiguousarray(zmask, dtype=np.uint64)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        out = ctypes.c_double()
        lib = self.ctx.lib
        A.raise_for(lib.sc_adjoint_forward(self.ctx.handle, n_qubits, ops, n_ops,
                                           p.ctypes.data_as(_dp), p.size, c.size,
                                           x.ctypes.data_as(_u64p), z.ctypes.data_as(_u64p),
                                           c.ctypes.data_as(_dp), ctypes.byref(out)), lib)
        self._n_params = p.size
        return out.value

    def backward(self) -> np.ndarray:
        grad = np.zeros(self._n_params)
        lib = self.ctx.lib
        A.raise_for(lib.sc_adjoint_backward(self.ctx.handle, grad.ctypes.data_as(_dp),
                                            grad.size), lib)
        return grad

    def value_and_grad(self, n_qubits, ops, n_ops, params, xmask, zmask, coeffs):
        e = self.forward(n_qubits, ops, n_ops, params, xmask, zmask, coeffs)
        return e, self.backward()

    def expectation(self, n_qubits, ops, n_ops, params, xmask, zmask, coeffs) -> float:
        """Forward only (used by finite-difference and parameter-shift baselines)."""
        return self.forward(n_qubits, ops, n_ops, params, xmask, zmask, coeffs)
