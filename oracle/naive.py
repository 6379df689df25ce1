"""CPU ORACLE -- TEST INFRASTRUCTURE ONLY.

Restatement of the reference's naive evaluator QuantumCircuit.apply
(core/.../quantum/QuantumCircuit.java:144-360): a ComplexNumber-by-ComplexNumber
loop over basis indices, the second oracle the reference's own engine tests
compare against at 1e-12 (StatevectorEngineTest.java:393-406).  Pure Python
loops, so it is meant for small circuits (a few qubits).
"""
from __future__ import annotations

from statecraft_b200 import quantum as Q


def _times(a: complex, b: complex) -> complex:
    # ComplexNumber.times (ComplexNumber.java:35-39)
    return complex(a.real * b.real - a.imag * b.imag, a.real * b.imag + a.imag * b.real)


def apply(circuit: Q.QuantumCircuit, initial=None) -> list[complex]:
    n = circuit.qubitCount
    dim = 1 << n
    if initial is None:
        state = [0j] * dim
        state[0] = 1 + 0j
    else:
        if len(initial) != dim:
            raise ValueError(f"Expected state vector of length {dim}, got {len(initial)}")
        state = [complex(x) if x is not None else 0j for x in initial]
    for op in circuit.operations:
        _apply_op(state, op)
    return state


def _apply_op(state: list, op) -> None:
    if isinstance(op, Q.SingleGateOperation):
        t = op.qubit
        g = op.gate
        g00, g01, g10, g11 = g.element(0, 0), g.element(0, 1), g.element(1, 0), g.element(1, 1)
        stride = 1 << t
        for base in range(0, len(state), stride << 1):
            for off in range(stride):
                i0, i1 = base + off, base + off + stride
                a0, a1 = state[i0], state[i1]
                state[i0] = _times(g00, a0) + _times(g01, a1)
                state[i1] = _times(g10, a0) + _times(g11, a1)
    elif isinstance(op, Q.CnotOperation):
        cm, tm = 1 << op.controlQubit, 1 << op.targetQubit
        for base in range(len(state)):
            if base & (cm | tm) == 0:
                i10, i11 = base | cm, base | cm | tm
                state[i10], state[i11] = state[i11], state[i10]
    elif isinstance(op, Q.TwoQubitGateOperation):
        fm, sm = 1 << op.firstQubit, 1 << op.secondQubit
        m = op.matrix
        for base in range(len(state)):
            if base & fm == 0 and base & sm == 0:
                idx = (base, base | sm, base | fm, base | fm | sm)
                a = [state[k] for k in idx]
                for r in range(4):
                    acc = _times(m[4 * r], a[0])
                    for c in range(1, 4):
                        acc = acc + _times(m[4 * r + c], a[c])
                    state[idx[r]] = acc
    elif isinstance(op, Q.TwoQubitDiagonalOperation):
        fm, sm = 1 << op.firstQubit, 1 << op.secondQubit
        d = op.diagonal
        for base in range(len(state)):
            if base & fm == 0 and base & sm == 0:
                idx = (base, base | sm, base | fm, base | fm | sm)
                for k in range(4):
                    state[idx[k]] = _times(d[k], state[idx[k]])
    elif isinstance(op, Q.SwapOperation):
        fm, sm = 1 << op.firstQubit, 1 << op.secondQubit
        for base in range(len(state)):
            if base & fm == 0 and base & sm == 0:
                state[base | sm], state[base | fm] = state[base | fm], state[base | sm]
    elif isinstance(op, Q.MultiControlOperation):
        tm = 1 << op.targetQubit
        cmask = 0
        for c in op.controlQubits:
            cmask |= 1 << c
        g = op.gate
        g00, g01, g10, g11 = g.element(0, 0), g.element(0, 1), g.element(1, 0), g.element(1, 1)
        for base in range(len(state)):
            if base & cmask == cmask and base & tm == 0:
                a0, a1 = state[base], state[base | tm]
                state[base] = _times(g00, a0) + _times(g01, a1)
                state[base | tm] = _times(g10, a0) + _times(g11, a1)
    elif isinstance(op, Q.MeasureOperation):
        raise NotImplementedError("Measurement operations cannot be evaluated using QuantumCircuit.apply")
    else:
        raise RuntimeError(f"Unsupported operation type: {type(op).__name__}")
