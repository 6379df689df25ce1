"""CPU tests of the native library: symbol exports, ABI layout, failure without a
GPU, and the fusion planner (order respects the dependency DAG; the plan encoding,
executed with the kernel's tile/stage semantics on the host, matches the oracle)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import randcirc as RCirc
from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import quantum as Q
from statecraft_b200.engine import serialize_circuit

HEADER = Path(__file__).resolve().parents[1] / "include" / "statecraft_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^SC_API\s+[\w\s\*]+?\b(sc_\w+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = A.load()
    syms = declared_symbols()
    assert len(syms) >= 19
    for name in syms:
        assert hasattr(lib, name), name
    assert set(syms) == set(A.SIGNATURES), "ctypes signature table out of sync with the header"


def test_abi_version_and_struct_sizes():
    lib = A.load()
    assert lib.sc_version() == A.SC_ABI_VERSION
    assert ctypes.sizeof(A.ScOp) == 280
    assert ctypes.sizeof(A.ScChannel) == 528
    assert ctypes.sizeof(A.ScConfig) == 40


def test_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = A.load()
    h = ctypes.c_void_p()
    rc = lib.sc_create(0, None, ctypes.byref(h))
    assert rc in (A.SC_ECUDA, A.SC_EINVAL)
    assert lib.sc_last_error()
    assert not h.value


def test_invalid_handle_rejected():
    lib = A.load()
    assert lib.sc_destroy(None) == A.SC_OK


def _plan_info(c, tile, low, nr, budget):
    ops, n_ops = serialize_circuit(c)
    order = np.zeros(max(1, n_ops), dtype=np.int64)
    cnt = [ctypes.c_int64() for _ in range(4)]
    k = A.load().sc_debug_plan_order(c.qubitCount, ops, n_ops, tile, low, nr, budget,
                                     order.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                     *[ctypes.byref(x) for x in cnt])
    assert k >= 0
    sweeps, stages, relayouts, restores = (x.value for x in cnt)
    return order[:k], dict(sweeps=sweeps, stages=stages, relayouts=relayouts, restores=restores)


def _plan_order(c, tile, low, nr, budget):
    order, info = _plan_info(c, tile, low, nr, budget)
    return order, info["sweeps"], info["stages"]


def _emulate(c, state, tile, low, nr, budget):
    ops, n_ops = serialize_circuit(c)
    st = state.copy()
    rc = A.load().sc_debug_emulate_sweeps(c.qubitCount, ops, n_ops, tile, low, nr, budget,
                                          st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc >= 0, A.load().sc_last_error()
    return st, rc


def _oracle(c, state):
    ops, n_ops = serialize_circuit(c)
    st = state.copy()
    rc, _ = O.run(c.qubitCount, ops, n_ops, st)
    assert rc == 0
    return st


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 11, 13])
@pytest.mark.parametrize("cfg", [(11, 4, 3, 96.0), (6, 2, 2, -1.0), (9, 5, 4, 24.0), (12, 3, 1, 8.0)])
def test_emulated_plan_matches_oracle(n, cfg):
    tile, low, nr, budget = cfg
    for seed in range(3):
        c = RCirc.random_circuit(n, 40, seed=1000 * n + seed)
        init = RCirc.random_state(n, seed)
        got, sweeps = _emulate(c, init, tile, low, nr, budget)
        want = _oracle(c, init)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def test_plan_order_is_a_permutation_and_respects_dependencies():
    c = RCirc.random_circuit(12, 300, seed=7)
    order, sweeps, stages = _plan_order(c, 11, 4, 3, 96.0)
    ops = c.operations
    assert sorted(order.tolist()) == list(range(len(ops)))
    # two ops keep their relative order when a qubit is touched by both and acted
    # on non-diagonally (as a target of a non-diagonal gate) by at least one
    pos = {int(o): k for k, o in enumerate(order)}
    for i in range(len(ops)):
        for j in range(i + 1, len(ops)):
            shared = (set(ops[i].qubits_touched()) & set(ops[j].qubits_touched()))
            if shared & (_dense_qubits(ops[i]) | _dense_qubits(ops[j])):
                assert pos[i] < pos[j], (i, j, ops[i], ops[j])


def _is_diag(gate) -> bool:
    return gate.element(0, 1) == 0 and gate.element(1, 0) == 0


def _dense_qubits(op) -> set:
    from statecraft_b200 import quantum as Q

    if isinstance(op, Q.SingleGateOperation):
        return set() if _is_diag(op.gate) else {op.qubit}
    if isinstance(op, Q.CnotOperation):
        return {op.targetQubit}
    if isinstance(op, Q.TwoQubitGateOperation):
        m = np.array(op.matrix).reshape(4, 4)
        return set() if np.count_nonzero(m - np.diag(np.diag(m))) == 0 else {op.firstQubit, op.secondQubit}
    if isinstance(op, Q.SwapOperation):
        return {op.firstQubit, op.secondQubit}
    if isinstance(op, Q.MultiControlOperation):
        return set() if _is_diag(op.gate) else {op.targetQubit}
    return set()


def test_brickwall_plan_uses_few_sweeps():
    from statecraft_b200 import workloads as W

    c = W.brickwall_circuit(20, 20, seed=2020, mcz=False, rzz=False)
    order, sweeps, stages = _plan_order(c, 11, 4, 3, -1.0)
    assert len(order) == len(c.operations)
    assert sweeps <= 3 * 20  # unfused would be 590 sweeps


@pytest.mark.parametrize("n,layers,cfg", [
    (16, 12, (8, 3, 3, -1.0)),
    (16, 12, (8, 4, 3, 40.0)),
    (17, 10, (9, 2, 2, -1.0)),
    (18, 8, (10, 4, 3, -1.0)),
])
def test_relayout_plans_match_oracle(n, layers, cfg):
    # brick-wall circuits move their working window along the chain: the planner
    # brings the next window's qubits onto the low physical bits between sweeps and
    # restores the identity layout at the end
    from statecraft_b200 import workloads as W

    c = W.brickwall_circuit(n, layers, seed=77 + n, mcz=False, rzz=True)
    _, info = _plan_info(c, *cfg)
    assert info["relayouts"] > 0
    init = RCirc.random_state(n, n)
    got, _ = _emulate(c, init, *cfg)
    np.testing.assert_allclose(got, _oracle(c, init), rtol=0, atol=1e-12)


def test_relayout_reduces_sweeps(monkeypatch):
    from statecraft_b200 import workloads as W

    c = W.brickwall_circuit(30, 40, seed=3030, mcz=False, rzz=False)
    _, with_layout = _plan_info(c, 10, 4, 3, -1.0)
    monkeypatch.setenv("STATECRAFT_B200_RELAYOUT", "0")
    _, without = _plan_info(c, 10, 4, 3, -1.0)
    assert without["relayouts"] == 0 and without["restores"] == 0
    assert with_layout["sweeps"] < 0.8 * without["sweeps"]


def test_rotation_form_scalar_stays_in_range():
    # 1-qubit gates in rotation form leave a scalar |u00| per gate that the sweeps
    # apply late; a long chain of near-pi rotations (|u00| = 0.06, just above the
    # 0.05 bound) would push the stored amplitudes past the double range without
    # the floor on that scalar
    from statecraft_b200 import quantum as Q

    n = 10
    theta = 2 * np.arccos(0.06)
    c = Q.QuantumCircuit(n)
    for q in range(n):
        c = c.append(Q.Hadamard(), q)
    rng = np.random.default_rng(6)
    for _ in range(400):
        q = int(rng.integers(0, n))
        c = c.append(Q.u3(theta, float(rng.uniform(0, 6.3)), float(rng.uniform(0, 6.3))), q)
        if rng.random() < 0.1:
            c = c.append(Q.CnotGate.of(), q, (q + 1) % n)
    init = RCirc.random_state(n, 3)
    for cfg in [(6, 2, 2, -1.0), (8, 3, 3, -1.0), (11, 4, 4, -1.0)]:
        got, _ = _emulate(c, init, *cfg)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, _oracle(c, init), rtol=0, atol=1e-12)


def test_runs_mixing_rotation_and_matrix_gates():
    # layers of u3 gates where some have |u00| below the rotation-form bound (0.05):
    # those take the rotation form as U X, so their record starts with an X on their
    # bits (folded into the stage's read where the record is the stage's only one)
    from statecraft_b200 import quantum as Q

    n = 12
    rng = np.random.default_rng(12)
    c = Q.QuantumCircuit(n)
    for layer in range(8):
        for q in range(n):
            u00 = 0.01 if rng.random() < 0.3 else float(rng.uniform(0.1, 1.0))
            c = c.append(Q.u3(2 * np.arccos(u00), float(rng.uniform(0, 6.3)),
                              float(rng.uniform(0, 6.3))), q)
        for q in range(layer % 2, n - 1, 2):
            c = c.append(Q.CnotGate.of(), q, q + 1)
    init = RCirc.random_state(n, 5)
    for cfg in [(11, 4, 4, -1.0), (8, 3, 3, -1.0), (6, 2, 2, -1.0)]:
        got, _ = _emulate(c, init, *cfg)
        np.testing.assert_allclose(got, _oracle(c, init), rtol=0, atol=1e-12)


@pytest.mark.parametrize("peephole", ["1", "0"])
@pytest.mark.parametrize("cfg", [(11, 4, 4, -1.0), (10, 4, 3, -1.0), (9, 3, 3, -1.0)])
def test_stage_peephole_matches_oracle(cfg, peephole, monkeypatch):
    # brick-wall layers with a multi-controlled Z and RZZ (the headline structure):
    # CNOTs with controls outside the registers become exit-slot folds, diagonals
    # move through register permutations and merge into rotation tables
    from statecraft_b200 import workloads as W

    monkeypatch.setenv("STATECRAFT_B200_PEEPHOLE", peephole)
    c = W.brickwall_circuit(17, 5, seed=1717, mcz=True, rzz=True)
    init = RCirc.random_state(17, 17)
    got, _ = _emulate(c, init, *cfg)
    np.testing.assert_allclose(got, _oracle(c, init), rtol=0, atol=1e-12)


def _with_slots(c, slots, paulis):
    """c with Pauli gates inserted after the ops named by slots (op index, qubit)."""
    gate = {1: Q.PauliX(), 2: Q.PauliY(), 3: Q.PauliZ()}
    out = Q.QuantumCircuit(c.qubitCount)
    k = 0
    for i, op in enumerate(c.operations):
        out = out._append(op)
        while k < len(slots) and slots[k][0] == i:
            if paulis[k]:
                out = out.append(gate[int(paulis[k])], slots[k][1])
            k += 1
    return out


def _emulate_slots(c, slots, paulis, state, tile, low, nr, budget):
    ops, n_ops = serialize_circuit(c)
    after = np.array([s[0] for s in slots], dtype=np.int64)
    qubit = np.array([s[1] for s in slots], dtype=np.int32)
    codes = np.ascontiguousarray(paulis, dtype=np.uint8)
    st = state.copy()
    rc = A.load().sc_debug_emulate_slots(
        c.qubitCount, ops, n_ops, tile, low, nr, budget,
        after.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
        qubit.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(slots),
        codes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
        st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc >= 0, A.load().sc_last_error()
    return st


def _ghz_chain(n, seed):
    from statecraft_b200 import workloads as W

    rng = np.random.default_rng(seed)
    c = W.ghz_circuit(n)
    for _ in range(3):  # more CNOT layers, mixed with rotations, as register permutations
        for q in rng.permutation(n - 1):
            c = c.append(Q.CnotGate.of(), int(q), int(q) + 1)
        c = c.append(RCirc.random_gate(rng), int(rng.integers(0, n)))
        c = c.appendSwap(int(rng.integers(0, n // 2)), int(rng.integers(n // 2, n)))
    return c


@pytest.mark.parametrize("peephole", ["1", "0"])
@pytest.mark.parametrize("cfg", [(11, 4, 4, -1.0), (10, 4, 3, -1.0), (9, 3, 2, 24.0)])
def test_pauli_slots_through_folded_permutations(cfg, peephole, monkeypatch):
    # noise slots after every op on each qubit it touches: CNOT chains fold into the
    # stage exit permutation and the slots after them are conjugated (X -> X^u,
    # Z -> +-Z^w, Y -> i X^u Z^w); one trajectory of every Pauli pattern mix
    monkeypatch.setenv("STATECRAFT_B200_PEEPHOLE", peephole)
    for n, seed in ((6, 1), (13, 2), (15, 3)):
        c = _ghz_chain(n, seed) if seed != 2 else RCirc.random_circuit(n, 60, seed=77)
        slots = []
        for i, op in enumerate(c.operations):
            for q in sorted(set(op.qubits_touched())):
                slots.append((i, int(q)))
        rng = np.random.default_rng(seed)
        init = RCirc.random_state(n, seed)
        for density in (0.05, 0.5):
            paulis = np.where(rng.random(len(slots)) < density,
                              rng.integers(1, 4, len(slots)), 0).astype(np.uint8)
            got = _emulate_slots(c, slots, paulis, init, *cfg)
            want = _oracle(_with_slots(c, slots, paulis), init)
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


@pytest.mark.parametrize("cfg", [(11, 4, 4, -1.0), (10, 4, 3, -1.0), (8, 3, 2, 24.0)])
def test_overlapping_permutation_folds(cfg, monkeypatch):
    # runs of CNOTs and swaps on the same register bits: folded permutations that
    # overlap compose into the exit permutation in time order
    monkeypatch.setenv("STATECRAFT_B200_PEEPHOLE", "1")
    for n, seed in ((9, 5), (14, 6), (16, 7)):
        c = RCirc.random_circuit(n, 120, seed=seed, kinds=["cnot", "cnot", "swap", "single"])
        init = RCirc.random_state(n, seed)
        got, _ = _emulate(c, init, *cfg)
        np.testing.assert_allclose(got, _oracle(c, init), rtol=0, atol=1e-12)


@pytest.mark.parametrize("dtype", [A.SC_C128, A.SC_C64])
@pytest.mark.parametrize("nr", [4, 3])
def test_exchange_tables_consistent_and_conflict_free(dtype, nr):
    # the shared-memory tables the sweep kernel gets: per exchange, every slot written
    # and read once, writer and reader agree on each amplitude's slot, and the
    # per-exchange swizzle leaves no 128-byte wavefront with a bank conflict
    from statecraft_b200 import workloads as W

    low = 4 if dtype == A.SC_C128 else 5
    circuits = [W.brickwall_circuit(26, 3, seed=26, mcz=True, rzz=True),
                RCirc.random_circuit(18, 150, seed=5),
                RCirc.random_circuit(14, 200, seed=9, kinds=["cnot", "swap", "single", "multi"])]
    for c in circuits:
        ops, n_ops = serialize_circuit(c)
        stats = np.zeros(4, dtype=np.int64)
        rc = A.load().sc_debug_check_exchanges(
            c.qubitCount, ops, n_ops, 11, low, nr, dtype,
            stats.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        assert rc > 0, A.load().sc_last_error()
        exchanges, general, wavefronts, conflicted = stats.tolist()
        assert exchanges > 0 and wavefronts > 0
        assert conflicted == 0


def test_exchange_tables_over_plan_shapes():
    # tile sizes, register counts and low-qubit counts the planner accepts, small
    # tiles (fewer threads than a wavefront) included: the tables stay consistent
    # and conflict-free for every shape
    checked = 0
    for seed, n in ((0, 7), (1, 13)):
        c = RCirc.random_circuit(n, 80, seed=100 * seed + n)
        ops, n_ops = serialize_circuit(c)
        for dtype in (A.SC_C128, A.SC_C64):
            for tile in (6, 8, 11):
                for nr in (2, 3, 4):
                    for low in (3, 4):
                        stats = np.zeros(4, dtype=np.int64)
                        rc = A.load().sc_debug_check_exchanges(
                            n, ops, n_ops, tile, low, nr, dtype,
                            stats.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
                        if rc < 0:  # a shape the planner does not take
                            assert b"inconsistent" not in (A.load().sc_last_error() or b"")
                            continue
                        assert stats[3] == 0, (n, dtype, tile, nr, low, stats.tolist())
                        checked += int(stats[0] > 0)
    assert checked >= 40


@pytest.mark.parametrize("dtype", [A.SC_C128, A.SC_C64])
def test_tile_tensor_boxes_match_tile_enumeration(dtype):
    # the whole-tile tensor copies (TMA boxes): every tile position is copied from the
    # amplitude the sweep's tile enumeration assigns to it, for single states and
    # batches, brick-wall (the headline's box shapes) and random plans
    from statecraft_b200 import workloads as W

    low = 4 if dtype == A.SC_C128 else 5
    cases = [(W.brickwall_circuit(26, 3, seed=26, mcz=True, rzz=True), 1),
             (W.brickwall_circuit(20, 2, seed=20, mcz=True, rzz=True), 3),
             (RCirc.random_circuit(18, 150, seed=5), 1),
             (W.ghz_circuit(16), 5),
             (RCirc.random_circuit(13, 90, seed=2), 7)]
    boxed = 0
    for c, batch in cases:
        ops, n_ops = serialize_circuit(c)
        stats = np.zeros(2, dtype=np.int64)
        rc = A.load().sc_debug_check_tile_tensors(
            c.qubitCount, ops, n_ops, 11, low, 4, dtype, batch,
            stats.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        assert rc > 0, A.load().sc_last_error()
        boxed += int(stats[0])
    assert boxed > 10


@pytest.mark.parametrize("fold", ["0", "1"])
@pytest.mark.parametrize("cfg", [(11, 4, 3, -1.0), (10, 4, 4, -1.0), (9, 3, 2, -1.0)])
def test_entry_folds_match_oracle(fold, cfg, monkeypatch):
    """Register permutations that open a stage are folded into its read (X, CNOT,
    SWAP, and X controlled from outside the registers, with per-thread flips); the
    emulated plan matches the oracle with the folds on and off, on circuits made of
    permutations between rotation layers."""
    monkeypatch.setenv("STATECRAFT_B200_ENTRY_FOLD", fold)
    tile, low, nr, budget = cfg
    for seed in range(3):
        n = 12
        c = RCirc.random_circuit(n, 120, seed=500 + seed,
                                 kinds=["single", "cnot", "swap", "multi", "cnot", "cnot"])
        # the plan does fold: records taken into stage reads, conditional ones among them
        ops, n_ops = serialize_circuit(c)
        st = np.zeros(3, dtype=np.int64)
        assert A.load().sc_debug_entry_folds(n, ops, n_ops, tile, low, nr, budget,
                                             st.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))) == A.SC_OK
        if fold == "1":
            assert st[1] > 0 and st[2] > 0, st
        else:
            assert st[1] == 0 and st[2] == 0, st
        init = RCirc.random_state(n, seed)
        got, _ = _emulate(c, init, tile, low, nr, budget)
        want = _oracle(c, init)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
