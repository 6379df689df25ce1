"""Parity at the sizes the benchmark configurations run, against the CPU oracle.

- 30 qubits, complex128: the headline brick-wall generator (U3 + CNOT brick + MCZ
  with 29 controls + RZZ on a seeded pair, angle seed 3030) for two layers, fused
  plan on the GPU; the full 2^30-amplitude state within 1e-12 max-abs of the
  oracle and countsAll(8192) with seed 42 identical outcome by outcome.  The
  reference's CDF is a left-to-right FP64 running sum over 2^30 entries
  (StatevectorEngine.java:314-323); the GPU reproduces that running sum bit for bit
  (integer effects of whole chunks inside one binade, exact adds elsewhere), so even
  draws within 1e-12 of an entry land where the reference puts them.  Reference
  rules: StatevectorEngineTest.java:393-406 (1e-12), StatevectorEngine.java:229-338
  (measurement).
- 26 qubits, complex128: the hardware-efficient ansatz of the adjoint workload
  (12 layers of RY, RZ and a CNOT ring, 624 angles, 64 random Pauli terms); <H>
  against the oracle, and the fused adjoint gradient on 8 angles against exact
  parameter shift and against central finite differences (h = 1e-6) on the plain
  forward engine, both within 1e-8.
- 22 qubits, complex64 with FP64 norms: the noisy-GHZ trajectory batch (a
  depolarizing channel with p = 1e-3 after every gate on every touched qubit), 32
  trajectories (noise seeds 43..74, where four trajectories take an X, Y or Z
  branch); branch choices identical to the oracle's state-dependent draws,
  states within 2e-5, and outcomes on shared uniforms identical except draws
  within the complex64 error band of a CDF boundary.

The 30-qubit case holds the oracle state (16 GiB) and the GPU state read back (16
GiB) in host memory; it runs only where the host has room for both.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import workloads as W
from statecraft_b200.adjoint import AdjointEngine
from statecraft_b200.engine import (B200Config, MeasurementInstruction, NativeContext,
                                    SimulationRequest, StatevectorB200Engine, serialize_channels,
                                    serialize_circuit)
from statecraft_b200.trajectories import run_trajectories, touched_qubit_depolarizing

pytestmark = pytest.mark.gpu

EPS = 1e-12
GIB = 1 << 30


def _host_bytes_available() -> int:
    try:
        import psutil

        return int(psutil.virtual_memory().available)
    except Exception:  # pragma: no cover - psutil is part of the image
        return int(os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE"))


def _max_abs_diff(a: np.ndarray, b: np.ndarray, chunk: int = 1 << 26) -> float:
    worst = 0.0
    for lo in range(0, a.size, chunk):
        worst = max(worst, float(np.max(np.abs(a[lo:lo + chunk] - b[lo:lo + chunk]))))
    return worst


def test_c2_30q_two_layers_state_and_counts_match_oracle():
    n, layers, shots, seed = 30, 2, 8192, 42
    if _host_bytes_available() < 40 * GIB:
        pytest.skip("the 30-qubit comparison needs about 40 GiB of free host memory")
    c = W.brickwall_circuit(n, layers, seed=3030, mcz=True, rzz=True)
    engine = StatevectorB200Engine(B200Config())
    try:
        req = (SimulationRequest.zeroState(c)
               .withMeasurement(MeasurementInstruction.countsAll(shots).withSeed(seed), False))
        hist = engine.simulate(req).measurement.counts
        ctx = engine.context()
        stats = ctx.plan_stats()
        assert stats["sweeps"] > 1  # the fused multi-sweep plan ran
        u = O.uniforms(seed, shots)
        gpu_out = ctx.sample(list(range(n)), shots, None, u)
        got = ctx.state(n)
    finally:
        engine.close()
    gpu_hist = {int(k): int(v) for k, v in zip(*np.unique(gpu_out, return_counts=True))}
    assert gpu_hist == hist  # the seeded path consumed SplittableRandom(42).nextDouble()

    ops, n_ops = serialize_circuit(c)
    want = O.initial_state(n)
    rc, _ = O.run(n, ops, n_ops, want)
    assert rc == 0
    diff = _max_abs_diff(got, want)
    del got
    assert diff <= EPS, diff

    # countsAll(8192) on the oracle with the same uniforms, outcome by outcome
    probs = O.probabilities(want, n, list(range(n)))
    del want
    cdf = O.cumulative(probs)
    del probs
    want_out = np.array([O.sample_outcome(cdf, float(x)) for x in u], dtype=np.int64)
    near = int(np.sum(np.abs(np.asarray(u)[:, None] - cdf[np.clip(
        np.searchsorted(cdf, u)[:, None] + np.array([-1, 0]), 0, cdf.size - 1)]).min(axis=1) < 1e-11))
    print("30q counts: %d of %d draws lie within 1e-11 of a CDF entry" % (near, shots))
    np.testing.assert_array_equal(gpu_out, want_out)


def test_c4_26q_adjoint_gradient_vs_shift_and_differences():
    n, layers, terms, h = 26, 12, 64, 1e-6
    ops, n_ops, n_params = W.hea_ops(n, layers)
    assert n_params == 624
    params = W.hea_params(n_params, seed=2626)
    x, z, c = W.random_pauli_sum(n, terms, seed=6464)
    eng = AdjointEngine()
    try:
        value, grad = eng.value_and_grad(n, ops, n_ops, params, x, z, c)
        picks = np.linspace(0, n_params - 1, 8).round().astype(int)
        shift = np.zeros(picks.size)
        fd = np.zeros(picks.size)
        for i, k in enumerate(picks):
            vals = []
            for s in (math.pi / 2, -math.pi / 2, h, -h):
                p = params.copy()
                p[k] += s
                vals.append(eng.expectation(n, ops, n_ops, p, x, z, c))
            shift[i] = 0.5 * (vals[0] - vals[1])
            fd[i] = (vals[2] - vals[3]) / (2 * h)
    finally:
        eng.close()
    print("26q adjoint: |grad - shift| = %.3e, |grad - FD| = %.3e"
          % (np.max(np.abs(grad[picks] - shift)), np.max(np.abs(grad[picks] - fd))))
    # random 64-term Pauli sums on 26 qubits have small gradients (about 1e-4)
    assert np.max(np.abs(grad[picks])) > 1e-5  # a gradient that is not trivially zero
    np.testing.assert_allclose(grad[picks], shift, rtol=0, atol=1e-8)
    np.testing.assert_allclose(grad[picks], fd, rtol=0, atol=1e-8)
    # <H> of the forward pass against the oracle's state
    st = O.initial_state(n)
    rc, _ = O.run(n, ops, n_ops, st, params=params)
    assert rc == 0
    assert value == pytest.approx(O.expect_pauli(st, n, x, z, c), abs=1e-11)


def test_c5_22q_complex64_trajectories_match_oracle():
    n, traj, shots, p = 22, 32, 64, 1e-3
    c = W.ghz_circuit(n)
    rec = touched_qubit_depolarizing(c, p)
    assert len(rec) == 43
    ctx = NativeContext(B200Config(dtype=A.SC_C64))
    try:
        res = run_trajectories(c, rec, traj, noise_seed=43, shots=shots, measure_seed=77,
                               return_states=True, context=ctx)
    finally:
        ctx.close()
    ops, n_ops = serialize_circuit(c)
    ch, n_ch = serialize_channels(rec)
    took = 0
    worst = 0.0
    mism = 0
    for t in range(traj):
        st = O.initial_state(n)
        rc, chosen = O.run(n, ops, n_ops, st, ch, n_ch, 43 + t)
        assert rc == 0
        np.testing.assert_array_equal(res.choices[t], chosen)
        took += int(np.count_nonzero(chosen))
        amp = st[0::2] + 1j * st[1::2]
        worst = max(worst, float(np.max(np.abs(res.states[t] - amp))))
        u = O.uniforms(77 + t, shots)
        cdf = O.cumulative(O.probabilities(st, n, list(range(n))))
        for k in range(shots):
            j = O.sample_outcome(cdf, float(u[k]))
            if j != res.outcomes[t, k]:
                edges = [cdf[j - 1] if j > 0 else 0.0, cdf[j]]
                assert min(abs(u[k] - e) for e in edges) < 1e-5
                mism += 1
    print("22q c64 trajectories: max |amp diff| = %.3e, noisy branches taken %d, "
          "outcome mismatches %d of %d" % (worst, took, mism, traj * shots))
    assert worst < 2e-5
    assert took > 0  # some trajectory left the identity branch
    assert mism <= 2
