"""Dense blocks on the FP64 tensor cores against the oracle.

Runs of gates that touch at most 5 qubits are composed on the host into one 2^k x
2^k unitary (k = 3..5) and applied by mma.sync FP64 tiles; the rest of the circuit
runs through the fused sweeps.  The blocks' threshold is forced low so every
eligible run becomes a block; states must match the oracle within 1e-12 (the
reference tests' EPS), as every other complex128 path does.
"""
import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200 import workloads as W
from statecraft_b200.engine import (B200Config, SimulationRequest, StatevectorB200Engine,
                                    serialize_circuit)

pytestmark = pytest.mark.gpu

EPS = 1e-12


@pytest.mark.parametrize("n", [8, 12, 16, 20])
def test_dense_blocks_match_oracle(n, monkeypatch):
    monkeypatch.setenv("STATECRAFT_B200_DENSE_BLOCKS", "1")
    c = W.dense_window_circuit(n, 6, seed=n)
    ops, n_ops = serialize_circuit(c)
    want = O.initial_state(n)
    rc, _ = O.run(n, ops, n_ops, want)
    assert rc == 0
    e = StatevectorB200Engine(B200Config(timing=True))
    try:
        got = e.simulate(SimulationRequest.zeroState(c)).finalState.data()
        stats = e.context().kernel_stats()
    finally:
        e.close()
    assert stats["block"]["launches"] > 0  # the tensor-core path ran
    np.testing.assert_allclose(got, want, rtol=0, atol=EPS)


def test_dense_blocks_off_and_on_agree(monkeypatch):
    n = 18
    c = W.dense_window_circuit(n, 9, seed=7)
    out = []
    for v in ("0", "1"):
        monkeypatch.setenv("STATECRAFT_B200_DENSE_BLOCKS", v)
        e = StatevectorB200Engine(B200Config())
        try:
            out.append(e.simulate(SimulationRequest.zeroState(c)).finalState.data())
        finally:
            e.close()
    np.testing.assert_allclose(out[0], out[1], rtol=0, atol=EPS)
