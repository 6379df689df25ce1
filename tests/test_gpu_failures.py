"""Failure detection on the GPU without a GPU fault.

- A tile copy that does not land: the sweep kernel's first wait of each CTA is put
  on a barrier that nothing arrives on (the STATECRAFT_B200_TEST_STALL_CYCLES hook,
  about 50 microseconds), so the bounded wait runs out; the kernel sets its error
  flag, stops waiting, drains the copies it issued (with the full bound) and
  returns; the host reports SC_ETIMEOUT, and the same context then runs the circuit
  correctly.
- Non-finite amplitudes: a NaN in the initial state reaches the Kraus branch
  weights of a noisy run and the total of the sampler, which the engine reports as
  IllegalStateException (StatevectorEngine.java:463-530, 590-600: invalid branch
  weights and norms are IllegalStateException).
"""
import math

import numpy as np
import pytest

import randcirc as RCirc
from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import quantum as Q
from statecraft_b200 import workloads as W
from statecraft_b200.engine import (B200Config, NativeContext, SimulationRequest,
                                    StatevectorB200Engine, serialize_circuit)
from statecraft_b200.noise import ErrorChannel, NoiseModel

pytestmark = pytest.mark.gpu


def test_stalled_tile_copy_reports_timeout_and_context_recovers(monkeypatch):
    n = 20
    c = W.brickwall_circuit(n, 2, seed=77, mcz=True, rzz=True)  # no layout change: tile copies
    ops, n_ops = serialize_circuit(c)
    ctx = NativeContext(B200Config())
    try:
        monkeypatch.setenv("STATECRAFT_B200_TEST_STALL_CYCLES", "100000")
        with pytest.raises(A.EngineError) as info:
            ctx.run_ops(n, ops, n_ops)
        assert info.value.status == A.SC_ETIMEOUT
        monkeypatch.delenv("STATECRAFT_B200_TEST_STALL_CYCLES")
        ctx.run_ops(n, ops, n_ops)
        got = ctx.state(n)
    finally:
        ctx.close()
    want = O.initial_state(n)
    rc, _ = O.run(n, ops, n_ops, want)
    assert rc == 0
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def _nan_state(n):
    st = RCirc.random_state(n, 4)
    st[2 * 5] = math.nan
    return st


def test_nan_state_in_noisy_run_raises_illegal_state():
    n = 6
    c = Q.QuantumCircuit(n).append(Q.Hadamard(), 0)
    model = NoiseModel.builder().afterAllGates(ErrorChannel.depolarizing(0.1, 0)).build()
    req = (SimulationRequest.withInitialState(c, Q.StateVector.fromArray(n, _nan_state(n)))
           .withNoiseModel(model).withNoiseSeed(3))
    e = StatevectorB200Engine(B200Config())
    try:
        with pytest.raises(A.IllegalStateException):
            e.simulate(req)
        # the context stays usable
        ok = e.simulate(SimulationRequest.zeroState(c)).finalState.data()
        assert ok[0] == pytest.approx(math.sqrt(0.5), abs=1e-15)
    finally:
        e.close()


def test_nan_state_sampling_raises_illegal_state():
    n = 10
    ctx = NativeContext(B200Config())
    try:
        ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), _nan_state(n))
        with pytest.raises(A.IllegalStateException):
            ctx.sample(list(range(n)), 64, 1)
    finally:
        ctx.close()
