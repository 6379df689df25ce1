"""Committed golden fixtures (tests/golden/goldens.json, written by
tests/golden/make_goldens.py from the oracle): the oracle must keep reproducing
them (CPU) and the GPU engine must match them (GPU)."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "goldens.json").read_text())


def test_oracle_reproduces_goldens():
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_goldens

    fresh = make_goldens.compute()
    b, g = fresh["brickwall12"], GOLD["brickwall12"]
    np.testing.assert_allclose(b["amplitudes_first16"], g["amplitudes_first16"], rtol=0, atol=1e-15)
    assert b["outcomes_first32"] == g["outcomes_first32"] and b["histogram"] == g["histogram"]
    np.testing.assert_allclose(fresh["qaoa"]["energies"], GOLD["qaoa"]["energies"], rtol=0, atol=1e-13)
    assert fresh["ghz_trajectories"]["choices"] == GOLD["ghz_trajectories"]["choices"]
    assert fresh["splitmix_doubles"]["values"] == GOLD["splitmix_doubles"]["values"]


@pytest.mark.gpu
def test_gpu_matches_goldens():
    from statecraft_b200 import workloads as W
    from statecraft_b200.batch import QaoaRingBatch
    from statecraft_b200.engine import (B200Config, MeasurementInstruction, SimulationRequest,
                                        StatevectorB200Engine)
    from statecraft_b200.trajectories import run_trajectories, touched_qubit_depolarizing

    g = GOLD["brickwall12"]
    c = W.brickwall_circuit(g["qubits"], g["layers"], seed=g["angle_seed"], mcz=True, rzz=True)
    eng = StatevectorB200Engine(B200Config())
    res = eng.simulate(SimulationRequest.zeroState(c).withMeasurement(
        MeasurementInstruction.samplesAll(g["shots"]).withSeed(g["seed"]), True))
    st = res.finalState.data()
    np.testing.assert_allclose(st[:32], g["amplitudes_first16"], rtol=0, atol=1e-12)
    p = st[0::2] ** 2 + st[1::2] ** 2
    assert abs(float(np.sum(np.arange(p.size) * p)) - g["sum_index_weighted_prob"]) < 1e-9
    # same uniforms on both sides; a draw within 1e-12 of a CDF boundary may differ
    got = list(res.measurement.outcomes[:32])
    assert sum(a != b for a, b in zip(got, g["outcomes_first32"])) <= 1
    eng.close()

    q = GOLD["qaoa"]
    b = W.qaoa_instances(len(q["n_qubits"]), q["layers"], q["seed"], n_min=4, n_max=9)
    batch = QaoaRingBatch(b.n_qubits, b.gammas, b.betas, tune=False)
    np.testing.assert_allclose(batch.evaluate(), q["energies"], rtol=0, atol=1e-10)
    batch.close()

    t = GOLD["ghz_trajectories"]
    ghz = W.ghz_circuit(t["qubits"])
    r = run_trajectories(ghz, touched_qubit_depolarizing(ghz, t["p"]), len(t["choices"]),
                         noise_seed=t["noise_seed"], shots=0, measure_seed=0)
    assert r.choices.tolist() == t["choices"]
