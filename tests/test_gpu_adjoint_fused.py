"""Fused adjoint reverse pass (dual-state sweeps with gradient probes) against the
gate-by-gate reverse pass and against parameter shift on the oracle.  Sizes start
at 16 qubits, where the reverse plan's tiles hold at least one warp per stage (the
fused path's range; smaller states take the gate-by-gate path)."""
import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import workloads as W
from statecraft_b200.adjoint import AdjointEngine
from statecraft_b200.engine import B200Config

pytestmark = pytest.mark.gpu


def grad(n, layers, seed, dtype=A.SC_C128, fused=True, monkeypatch=None):
    ops, n_ops, n_params = W.hea_ops(n, layers)
    params = W.hea_params(n_params, seed)
    x, z, c = W.random_pauli_sum(n, 12, seed + 1)
    monkeypatch.setenv("STATECRAFT_B200_ADJOINT_FUSED", "1" if fused else "0")
    eng = AdjointEngine(B200Config(dtype=dtype))
    try:
        value, g = eng.value_and_grad(n, ops, n_ops, params, x, z, c)
    finally:
        eng.close()
    return value, np.asarray(g), (ops, n_ops, params, x, z, c)


@pytest.mark.parametrize("n,layers", [(16, 3), (18, 2), (20, 2)])
def test_fused_matches_gate_by_gate(n, layers, monkeypatch):
    v1, g1, _ = grad(n, layers, 100 + n, fused=True, monkeypatch=monkeypatch)
    v0, g0, _ = grad(n, layers, 100 + n, fused=False, monkeypatch=monkeypatch)
    assert abs(v1 - v0) < 1e-12
    np.testing.assert_allclose(g1, g0, rtol=0, atol=1e-11)
    assert np.max(np.abs(g0)) > 1e-3  # a gradient that is not trivially zero


def test_fused_matches_parameter_shift(monkeypatch):
    n = 16
    _, g, (ops, n_ops, params, x, z, c) = grad(n, 2, 7, fused=True, monkeypatch=monkeypatch)
    shift = np.zeros(len(params))
    for k in range(len(params)):
        vals = []
        for sgn in (1, -1):
            p = params.copy()
            p[k] += sgn * np.pi / 2
            st = O.initial_state(n)
            rc, _ = O.run(n, ops, n_ops, st, params=p)
            assert rc == 0
            vals.append(O.expect_pauli(st, n, x, z, c))
        shift[k] = 0.5 * (vals[0] - vals[1])
    np.testing.assert_allclose(g, shift, rtol=0, atol=1e-8)


def test_fused_complex64(monkeypatch):
    _, g64, _ = grad(18, 2, 55, dtype=A.SC_C64, fused=True, monkeypatch=monkeypatch)
    _, g128, _ = grad(18, 2, 55, fused=True, monkeypatch=monkeypatch)
    assert np.max(np.abs(g64 - g128)) < 1e-4


def test_backward_after_another_run_is_rejected():
    # the backward pass starts from the forward pass's state and lambda: a run on the
    # same context in between replaces the state, so backward must refuse
    from statecraft_b200.engine import serialize_circuit

    ops, n_ops, n_params = W.hea_ops(10, 1)
    params = W.hea_params(n_params, 3)
    x, z, c = W.random_pauli_sum(10, 4, 4)
    eng = AdjointEngine()
    try:
        eng.forward(10, ops, n_ops, params, x, z, c)
        other, n_other = serialize_circuit(W.brickwall_circuit(10, 1, seed=5))
        eng.ctx.run_ops(10, other, n_other)
        with pytest.raises(A.IllegalStateException, match="preceding sc_adjoint_forward"):
            eng.backward()
    finally:
        eng.close()


def _mixed_ops(n, seed):
    """RX / RY / RZ parameters among fixed 1-qubit gates (H, S, a general unitary,
    real rotations carrying a phase, some past pi/2) and CNOTs: the reverse plan
    has lifted rotations, half diagonals and matrix records side by side."""
    rng = np.random.default_rng(seed)
    ops = []
    p = 0

    def single(q, u):
        ops.append((A.SC_OP_SINGLE, q, -1, -1, u))

    h = np.array([[1, 1], [1, -1]], dtype=complex) / np.sqrt(2)
    s_gate = np.diag([1, 1j])
    for layer in range(3):
        for q in range(n):
            kind = (A.SC_OP_RX, A.SC_OP_RY, A.SC_OP_RZ)[(q + layer) % 3]
            ops.append((kind, q, -1, p, None))
            p += 1
            r = rng.integers(4)
            if r == 0:
                single(q, h)
            elif r == 1:
                single(q, s_gate)
            elif r == 2:
                al = rng.uniform(-np.pi, np.pi)
                single(q, np.exp(1j * rng.uniform(0, 2 * np.pi)) *
                       np.array([[np.cos(al), -np.sin(al)], [np.sin(al), np.cos(al)]]))
            else:
                a, b, c = rng.uniform(0, 2 * np.pi, 3)
                single(q, np.array([[np.cos(a / 2), -np.exp(1j * c) * np.sin(a / 2)],
                                    [np.exp(1j * b) * np.sin(a / 2),
                                     np.exp(1j * (b + c)) * np.cos(a / 2)]]))
        for q in range(layer % 2, n - 1, 2):
            ops.append((A.SC_OP_CNOT, q, q + 1, -1, None))
    arr = (A.ScOp * len(ops))()
    for i, (kind, q0, q1, param, u) in enumerate(ops):
        arr[i].kind, arr[i].q0, arr[i].q1, arr[i].param = kind, q0, q1, param
        if u is not None:
            for k, z in enumerate(np.asarray(u).reshape(-1)):
                arr[i].m[2 * k], arr[i].m[2 * k + 1] = z.real, z.imag
    return arr, len(ops), p


@pytest.mark.parametrize("n", [16, 18])
def test_fused_mixed_gates_match_gate_by_gate(n, monkeypatch):
    ops, n_ops, n_params = _mixed_ops(n, 300 + n)
    params = W.hea_params(n_params, 17 + n)
    x, z, c = W.random_pauli_sum(n, 10, 40 + n)
    out = []
    for fused in (True, False):
        monkeypatch.setenv("STATECRAFT_B200_ADJOINT_FUSED", "1" if fused else "0")
        eng = AdjointEngine(B200Config())
        try:
            v, g = eng.value_and_grad(n, ops, n_ops, params, x, z, c)
        finally:
            eng.close()
        out.append((v, np.asarray(g)))
    assert abs(out[0][0] - out[1][0]) < 1e-12
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=0, atol=1e-11)
    assert np.max(np.abs(out[1][1])) > 1e-3
