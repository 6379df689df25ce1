"""The comparison runner on the GPU, started the way the benchmark harness starts a
runner (a subprocess printing one JSON line): schema, noiseless amplitudes and
noisy trajectory averages against the same protocol run on the oracle."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import test_comparison as TC
from statecraft_b200 import comparison as C

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def run_module(args):
    out = subprocess.run([sys.executable, "-m", "statecraft_b200.comparison", *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return TC.check_schema(out.stdout.strip().splitlines()[-1])


def oracle_result(args):
    opts = C.parse_options(args)
    from statecraft_b200.engine import SimulationRequest
    return C.run_fixture(opts, TC.OracleEngine(), SimulationRequest)


GHZ5 = {"qubits": 5, "operations": [{"gate": "h", "target": 0}] +
        [{"gate": "cx", "control": k, "target": k + 1} for k in range(4)] +
        [{"gate": "cp", "control": 4, "target": 0, "angle": 0.7}, {"gate": "measure"}]}


def test_ideal_fixture_matches_oracle(tmp_path):
    args = ["--fixture-id", "ghz5", "--category", "ideal", "--circuit-json",
            TC.write(tmp_path, GHZ5), "--warmup-runs", "1", "--timed-runs", "3"]
    got, want = run_module(args), oracle_result(args)
    assert got["operations"] == 6 and got["qubits"] == 5 and len(got["timed_runs_ms"]) == 3
    np.testing.assert_allclose(got["probabilities"], want["probabilities"], rtol=0, atol=1e-12)
    sv = np.array(got["statevector"]).reshape(-1)
    np.testing.assert_allclose(sv, want["statevector"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("noise", [
    ["--noise-type", "phase_flip", "--noise-probability", "0.06", "--noise-qubits", "0,1"],
    ["--noise-type", "amplitude_damping", "--noise-gamma", "0.04", "--noise-qubits", "0,1"],
    ["--noise-type", "phase_damping", "--noise-lambda", "0.05", "--noise-qubits", "0,1,2"],
])
def test_noisy_fixture_matches_oracle(tmp_path, noise):
    args = ["--fixture-id", "noisy", "--category", "noise", "--circuit-json",
            TC.write(tmp_path, GHZ5), "--warmup-runs", "1", "--timed-runs", "1",
            "--noise-trajectories", "64", "--noise-seed", "91003", *noise]
    got, want = run_module(args), oracle_result(args)
    assert "statevector" not in got and got["noise_trajectories"] == 64
    np.testing.assert_allclose(got["probabilities"], want["probabilities"], rtol=0, atol=1e-12)
