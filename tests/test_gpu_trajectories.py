"""Batched noisy trajectories on the GPU against the oracle's per-trajectory runs.

The oracle runs each trajectory like StatevectorEngine.simulate: state-dependent
Kraus branch weights, one nextDouble(total) per noise record from
SplittableRandom(noise_seed + t), renormalisation.  Bars: identical branch choices;
final states within 1e-12 (complex128) / 2e-5 (complex64) max-abs; outcome
histograms identical when both sides sample the same uniforms, and within the
total-variation bound max(0.01, 3 x TV between two disjoint-seed oracle batches).
"""
import numpy as np
import pytest

import randcirc as RCirc
from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import noise as N
from statecraft_b200 import workloads as W
from statecraft_b200.engine import B200Config, NativeContext, serialize_channels, serialize_circuit
from statecraft_b200.trajectories import (run_trajectories, total_variation,
                                          touched_qubit_depolarizing)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = NativeContext(B200Config())
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx64():
    c = NativeContext(B200Config(dtype=A.SC_C64))
    yield c
    c.close()


def _oracle_trajectory(circuit, records, seed):
    n = circuit.qubitCount
    ops, n_ops = serialize_circuit(circuit)
    ch, n_ch = serialize_channels(records)
    st = O.initial_state(n)
    rc, chosen = O.run(n, ops, n_ops, st, ch, n_ch, seed)
    assert rc == 0
    return st[0::2] + 1j * st[1::2], chosen


@pytest.mark.parametrize("n,p", [(6, 0.3), (9, 0.1)])
def test_ghz_choices_and_states_match_oracle(ctx, n, p):
    c = W.ghz_circuit(n)
    rec = touched_qubit_depolarizing(c, p)
    res = run_trajectories(c, rec, 24, noise_seed=1000, shots=0, measure_seed=0,
                           return_states=True, context=ctx)
    for t in range(24):
        want, chosen = _oracle_trajectory(c, rec, 1000 + t)
        np.testing.assert_array_equal(res.choices[t], chosen)
        np.testing.assert_allclose(res.states[t], want, rtol=0, atol=1e-12)
    assert np.count_nonzero(res.choices) > 0  # some trajectories took Pauli branches


def test_random_circuits_with_pauli_noise(ctx):
    # dense gates, controlled gates and swaps with noise slots inside fused plans
    for seed in range(3):
        n = 11
        c = RCirc.random_circuit(n, 60, seed=300 + seed)
        rec = touched_qubit_depolarizing(c, 0.05)
        res = run_trajectories(c, rec, 6, noise_seed=77 * seed, shots=0, measure_seed=0,
                               return_states=True, context=ctx)
        for t in range(6):
            want, chosen = _oracle_trajectory(c, rec, 77 * seed + t)
            np.testing.assert_array_equal(res.choices[t], chosen)
            np.testing.assert_allclose(res.states[t], want, rtol=0, atol=1e-12)


def test_permutation_ladders_with_dense_noise(ctx):
    # CNOT ladders and swaps fold into the stage exit permutations and the Pauli
    # slots after them run conjugated (i^p X^u Z^w); heavy noise so most slots in
    # most trajectories take an X, Y or Z branch
    from statecraft_b200 import quantum as Q

    n = 14
    rng = np.random.default_rng(14)
    c = W.ghz_circuit(n)
    for _ in range(3):
        for q in rng.permutation(n - 1):
            c = c.append(Q.CnotGate.of(), int(q), int(q) + 1)
        c = c.appendSwap(int(rng.integers(0, n // 2)), int(rng.integers(n // 2, n)))
        c = c.append(RCirc.random_gate(rng), int(rng.integers(0, n)))
    rec = touched_qubit_depolarizing(c, 0.5)
    res = run_trajectories(c, rec, 8, noise_seed=4242, shots=0, measure_seed=0,
                           return_states=True, context=ctx)
    for t in range(8):
        want, chosen = _oracle_trajectory(c, rec, 4242 + t)
        np.testing.assert_array_equal(res.choices[t], chosen)
        np.testing.assert_allclose(res.states[t], want, rtol=0, atol=1e-12)
    assert np.count_nonzero(res.choices) > len(rec) * 8 // 4


def test_complex64_trajectories(ctx64):
    c = W.ghz_circuit(10)
    rec = touched_qubit_depolarizing(c, 0.2)
    res = run_trajectories(c, rec, 8, noise_seed=5, shots=0, measure_seed=0,
                           return_states=True, context=ctx64)
    for t in range(8):
        want, chosen = _oracle_trajectory(c, rec, 5 + t)
        np.testing.assert_array_equal(res.choices[t], chosen)
        np.testing.assert_allclose(res.states[t], want, rtol=0, atol=2e-5)


def test_histograms_match_oracle(ctx):
    n, traj, shots = 12, 96, 64
    c = W.ghz_circuit(n)
    rec = touched_qubit_depolarizing(c, 0.02)
    res = run_trajectories(c, rec, traj, noise_seed=4242, shots=shots, measure_seed=99,
                           context=ctx)
    oracle_out = []
    for t in range(traj):
        amp, _ = _oracle_trajectory(c, rec, 4242 + t)
        st = np.empty(2 << n)
        st[0::2], st[1::2] = amp.real, amp.imag
        oracle_out.append(O.sample(st, n, list(range(n)), shots, 99 + t))
    oracle_out = np.array(oracle_out)
    # same uniforms on both sides: the outcomes agree except draws within 1e-12 of a
    # CDF boundary (the two prefix sums round differently)
    assert np.count_nonzero(res.outcomes != oracle_out) <= 2
    # the total-variation bound against an oracle batch with disjoint seeds
    other = []
    for t in range(traj):
        amp, _ = _oracle_trajectory(c, rec, 90000 + t)
        st = np.empty(2 << n)
        st[0::2], st[1::2] = amp.real, amp.imag
        other.append(O.sample(st, n, list(range(n)), shots, 7000 + t))
    h_gpu = res.histogram()
    h_or = dict(zip(*np.unique(oracle_out, return_counts=True)))
    h_other = dict(zip(*np.unique(np.array(other), return_counts=True)))
    assert total_variation(h_gpu, h_or) <= max(0.01, 3 * total_variation(h_or, h_other))


def _channel_records(circuit, channels):
    """channels[k % len] after gate k, on every qubit the gate touches (a tuple entry:
    each of its channels in turn on each qubit)"""
    out = []
    from statecraft_b200 import quantum as Q
    for i, op in enumerate(circuit.operations):
        if isinstance(op, Q.MeasureOperation):
            continue
        chan = channels[i % len(channels)]
        if chan is None:
            continue
        for q in sorted(op.qubits_touched()):
            for ch in (chan if isinstance(chan, tuple) else (chan,)):
                kraus = tuple(np.array(k.matrix, dtype=complex).reshape(2, 2)
                              for k in ch.krausDecomposition())
                out.append(N.FlatChannel(i, q, kraus))
    return out


_CHANNELS = {
    "amplitude_damping": [N.AmplitudeDampingChannel(0.2, (0,))],
    "phase_damping": [N.PhaseDampingChannel(0.3, (0,))],
    "thermal": [N.ThermalRelaxationChannel(50.0, 70.0, 9.0, (0,))],
    "mixed": [N.AmplitudeDampingChannel(0.15, (0,)), N.DepolarizingChannel(0.2, (0,)), None,
              N.PhaseDampingChannel(0.25, (0,)), N.PhaseFlipChannel(0.3, (0,))],
    # two state-dependent records on the same qubit back to back
    "stacked": [(N.AmplitudeDampingChannel(0.2, (0,)), N.PhaseDampingChannel(0.2, (0,))),
                (N.DepolarizingChannel(0.1, (0,)), N.AmplitudeDampingChannel(0.25, (0,)))],
}


@pytest.mark.parametrize("kind", sorted(_CHANNELS))
def test_state_dependent_channels_match_oracle(ctx, kind):
    # records whose branch weights depend on the state end a fused segment; their
    # weights, draws and K / sqrt(w) run on the device for every trajectory
    n, traj = 9, 12
    c = RCirc.random_circuit(n, 40, seed=910)
    rec = _channel_records(c, _CHANNELS[kind])
    # records after gates on three or more qubits (multi-controlled gates) included
    assert max(len(op.qubits_touched()) for op in c.operations) >= 3
    res = run_trajectories(c, rec, traj, noise_seed=313, shots=0, measure_seed=0,
                           return_states=True, context=ctx)
    for t in range(traj):
        want, chosen = _oracle_trajectory(c, rec, 313 + t)
        np.testing.assert_array_equal(res.choices[t], chosen)
        np.testing.assert_allclose(res.states[t], want, rtol=0, atol=1e-12)
    assert np.count_nonzero(res.choices) > 0


def test_state_dependent_channels_complex64(ctx64):
    c = W.ghz_circuit(10)
    rec = _channel_records(c, [N.AmplitudeDampingChannel(0.3, (0,))])
    res = run_trajectories(c, rec, 8, noise_seed=21, shots=0, measure_seed=0,
                           return_states=True, context=ctx64)
    for t in range(8):
        want, chosen = _oracle_trajectory(c, rec, 21 + t)
        np.testing.assert_array_equal(res.choices[t], chosen)
        np.testing.assert_allclose(res.states[t], want, rtol=0, atol=2e-5)


def test_graph_replay_and_seeds(ctx):
    # the second call with the same circuit replays the captured graph; new seeds
    # reach its kernels through device memory; a timed (eager) context agrees
    n, traj, shots = 11, 40, 32
    c = W.ghz_circuit(n)
    rec = _channel_records(c, [N.AmplitudeDampingChannel(0.1, (0,)), N.DepolarizingChannel(0.05, (0,))])
    a = run_trajectories(c, rec, traj, noise_seed=5, shots=shots, measure_seed=6, context=ctx)
    info = ctx.trajectories_info()
    assert info["graph"] == 1
    b = run_trajectories(c, rec, traj, noise_seed=5, shots=shots, measure_seed=6, context=ctx)
    np.testing.assert_array_equal(a.outcomes, b.outcomes)
    np.testing.assert_array_equal(a.choices, b.choices)
    d = run_trajectories(c, rec, traj, noise_seed=500, shots=shots, measure_seed=600,
                         return_states=True, context=ctx)
    for t in range(0, traj, 7):
        want, chosen = _oracle_trajectory(c, rec, 500 + t)
        np.testing.assert_array_equal(d.choices[t], chosen)
        np.testing.assert_allclose(d.states[t], want, rtol=0, atol=1e-12)
    timed = NativeContext(B200Config(timing=True))
    try:
        e = run_trajectories(c, rec, traj, noise_seed=5, shots=shots, measure_seed=6, context=timed)
        assert timed.trajectories_info()["graph"] == 0
    finally:
        timed.close()
    np.testing.assert_array_equal(a.outcomes, e.outcomes)
    np.testing.assert_array_equal(a.choices, e.choices)


def test_autotuned_shape_matches_oracle():
    tuned = NativeContext(B200Config(autotune=True))
    try:
        n = 14
        c = RCirc.random_circuit(n, 50, seed=14)
        rec = touched_qubit_depolarizing(c, 0.05)
        res = run_trajectories(c, rec, 6, noise_seed=9, shots=0, measure_seed=0,
                               return_states=True, context=tuned)
        info = tuned.trajectories_info()
        assert info["tuned_ms"] > 0.0 and info["tile_qubits"] > 0
        for t in range(6):
            want, chosen = _oracle_trajectory(c, rec, 9 + t)
            np.testing.assert_array_equal(res.choices[t], chosen)
            np.testing.assert_allclose(res.states[t], want, rtol=0, atol=1e-12)
    finally:
        tuned.close()


def test_invalid_weights_raise_illegal_state(ctx):
    from statecraft_b200 import quantum as Q

    c = Q.QuantumCircuit(4).append(Q.PauliZ(), 1)
    # a Pauli record with zero weight (the host draw) and a projector onto |1> of a
    # qubit in |0> (weights summed on the device, total 0): both IllegalStateException
    zero = (np.zeros((2, 2), dtype=complex),)
    proj = (np.array([[0, 0], [0, 1]], dtype=complex),)
    for kraus in (zero, proj):
        with pytest.raises(A.IllegalStateException):
            run_trajectories(c, [N.FlatChannel(0, 0, kraus)], 4, noise_seed=1, shots=8,
                             measure_seed=1, context=ctx)
    # the context still runs batches
    ok = run_trajectories(W.ghz_circuit(4), [], 2, noise_seed=1, shots=4, measure_seed=1,
                          context=ctx)
    assert set(np.unique(ok.outcomes)) <= {0, 15}
