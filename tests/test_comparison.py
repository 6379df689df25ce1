"""Comparison runner (statecraft_b200/comparison.py): arguments, number format and
result schema of StatecraftComparisonRunner.java, and its run protocol (warm-up and
timed runs, noise seeds noise_seed + t, averaged trajectory probabilities) driven
through a stand-in engine built on the oracle, so it runs without a GPU."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200 import comparison as C
from statecraft_b200 import noise as N
from statecraft_b200 import quantum as Q
from statecraft_b200.engine import SimulationRequest, serialize_channels, serialize_circuit

BELL = {"qubits": 2, "operations": [{"gate": "h", "target": 0},
                                    {"gate": "cx", "control": 0, "target": 1}]}


class OracleEngine:
    """Test stand-in for StatevectorB200Engine.simulate on the oracle."""

    def __init__(self):
        self.seeds = []

    def simulate(self, req):
        c = req.circuit
        ops, n_ops = serialize_circuit(c)
        st = O.initial_state(c.qubitCount)
        if req.noiseModel is not None:
            ch, n_ch = serialize_channels(N.flatten_schedule(c, req.noiseModel))
            self.seeds.append(req.noiseSeed)
            rc, _ = O.run(c.qubitCount, ops, n_ops, st, ch, n_ch, req.noiseSeed)
        else:
            rc, _ = O.run(c.qubitCount, ops, n_ops, st)
        assert rc == 0

        class R:
            finalState = Q.StateVector.fromArray(c.qubitCount, st)
        return R()


def write(tmp_path, circuit) -> str:
    p = tmp_path / "fixture.statecraft.json"
    p.write_text(json.dumps(circuit))
    return str(p)


def check_schema(line: str) -> dict:
    # the checks of the harness's validate_result_schema (comparison_lib.py:193-204)
    r = json.loads(line)
    for field in ("runner", "fixture_id", "category", "status", "timed_runs_ms", "mean_ms",
                  "probabilities"):
        assert field in r
    assert r["status"] == "ok" and r["runner"] == "statecraft"
    assert isinstance(r["timed_runs_ms"], list) and isinstance(r["probabilities"], list)
    return r


def test_options_defaults_and_requirements():
    o = C.parse_options(["--circuit-json", "x.json"])
    assert (o.warmup_runs, o.timed_runs, o.parallelism, o.noise_trajectories) == (1, 5, 1, 512)
    assert o.noise_seed == 0x51A7EC0FFEEA and o.noise_type is None
    o = C.parse_options(["--circuit-json", "x", "--noise-type", "phase_flip", "--noise-qubits", "0, 2"])
    assert o.noise_qubits == [0, 2]
    with pytest.raises(SystemExit):
        C.parse_options(["--fixture-id", "a"])
    with pytest.raises(SystemExit):
        C.parse_options(["--circuit-json", "x", "--noise-type", "depolarizing"])
    with pytest.raises(ValueError, match="unknown noise type"):
        C.noise_model(C.parse_options(["--circuit-json", "x", "--noise-type", "bitflop",
                                       "--noise-qubits", "0"]))


def test_java_number_format():
    assert C.java_g17(0.5) == "0.50000000000000000"
    assert C.java_g17(1e-20) == "1.0000000000000000e-20"
    assert C.java_g17(0.0) == "0.0000000000000000"
    assert C.java_g17(-2.0) == "-2.0000000000000000"
    assert C.java_g17(123456.789) == "123456.78900000000"
    assert C.java_g17(0.1) == "0.10000000000000000"
    assert C.java_g17(1e16) == "10000000000000000"
    assert C.java_g17(1e17) == "1.0000000000000000e+17"
    assert C.java_g17(-0.0) == "-0.0000000000000000"
    for x in (1 / 3, 2 ** -0.5, 5e-324, 1.7976931348623157e308, 9.9999e-5, 1e-4):
        assert float(C.java_g17(x)) == x


def test_noiseless_fixture(tmp_path, capsys):
    eng = OracleEngine()
    C.main(["--fixture-id", "bell", "--category", "ideal", "--circuit-json", write(tmp_path, BELL),
            "--warmup-runs", "2", "--timed-runs", "3"], engine_factory=lambda: eng)
    r = check_schema(capsys.readouterr().out.strip())
    assert (r["fixture_id"], r["qubits"], r["operations"], r["timed_runs"]) == ("bell", 2, 2, 3)
    assert len(r["timed_runs_ms"]) == 3 and r["noise_trajectories"] == 0
    np.testing.assert_allclose(r["probabilities"], [0.5, 0, 0, 0.5], atol=1e-15)
    sv = np.array(r["statevector"])
    np.testing.assert_allclose(sv[[0, 3], 0], [2 ** -0.5] * 2, atol=1e-15)


@pytest.mark.parametrize("noise", [
    ["--noise-type", "depolarizing", "--noise-probability", "0.08", "--noise-qubits", "0"],
    ["--noise-type", "amplitude_damping", "--noise-gamma", "0.3", "--noise-qubits", "0,1"],
    ["--noise-type", "thermal_relaxation", "--noise-t1", "5e-5", "--noise-t2", "3e-5",
     "--noise-gate-time", "1e-5", "--noise-qubits", "1"],
])
def test_noisy_fixture_averages_seeded_trajectories(tmp_path, capsys, noise):
    eng = OracleEngine()
    C.main(["--fixture-id", "n", "--category", "noise", "--circuit-json", write(tmp_path, BELL),
            "--warmup-runs", "1", "--timed-runs", "2", "--noise-trajectories", "16",
            "--noise-seed", "91000", *noise], engine_factory=lambda: eng)
    r = check_schema(capsys.readouterr().out.strip())
    assert "statevector" not in r and r["noise_trajectories"] == 16
    # warm-up run seed, then two timed runs over seeds 91000..91015
    assert eng.seeds == [91000] + list(range(91000, 91016)) * 2
    opts = C.parse_options(["--circuit-json", "x", *noise])
    model = C.noise_model(opts)
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
    want = np.zeros(4)
    for t in range(16):
        st = OracleEngine().simulate(
            SimulationRequest.zeroState(c).withNoiseModel(model).withNoiseSeed(91000 + t)).finalState.data()
        want += st[0::2] ** 2 + st[1::2] ** 2
    np.testing.assert_allclose(r["probabilities"], want / 16, rtol=0, atol=1e-15)
