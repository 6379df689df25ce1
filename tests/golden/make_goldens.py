"""Writes tests/golden/goldens.json: small fixed cases computed on the CPU oracle.

The oracle restates the reference engine (oracle/sc_oracle.c) and is itself pinned
against the reference's own tests (tests/test_oracle_pins.py).  These fixtures
freeze its outputs for a few seeded workloads so that both the oracle (CPU tests)
and the GPU engine (GPU tests) are checked against the same committed numbers.

    python tests/golden/make_goldens.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def compute() -> dict:
    from oracle import oracle as O
    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import serialize_channels, serialize_circuit
    from statecraft_b200.trajectories import touched_qubit_depolarizing

    out = {}
    # brick-wall (the C1 generator at 12 qubits, 6 layers, MCZ + RZZ), countsAll(256) seed 42
    n = 12
    c = W.brickwall_circuit(n, 6, seed=2020, mcz=True, rzz=True)
    ops, n_ops = serialize_circuit(c)
    st = O.initial_state(n)
    assert O.run(n, ops, n_ops, st)[0] == 0
    outc = O.sample(st, n, list(range(n)), 256, 42)
    out["brickwall12"] = {
        "qubits": n, "layers": 6, "angle_seed": 2020, "shots": 256, "seed": 42,
        "amplitudes_first16": st[:32].tolist(),
        "sum_index_weighted_prob": float(np.sum(np.arange(1 << n) * (st[0::2] ** 2 + st[1::2] ** 2))),
        "outcomes_first32": outc[:32].tolist(),
        "histogram": {str(k): int(v) for k, v in zip(*np.unique(outc, return_counts=True))},
    }
    # QAOA ring energies
    b = W.qaoa_instances(8, 3, 99, n_min=4, n_max=9)
    out["qaoa"] = {
        "seed": 99, "layers": 3, "n_qubits": b.n_qubits.tolist(),
        "energies": [O.qaoa_ring_energy(int(k), b.gammas[i], b.betas[i])
                     for i, k in enumerate(b.n_qubits)],
    }
    # noisy GHZ trajectories: branch choices per trajectory
    g = W.ghz_circuit(6)
    rec = touched_qubit_depolarizing(g, 0.3)
    gops, g_n = serialize_circuit(g)
    ch, n_ch = serialize_channels(rec)
    choices = []
    for t in range(6):
        s2 = O.initial_state(6)
        rc, chosen = O.run(6, gops, g_n, s2, ch, n_ch, 500 + t)
        assert rc == 0
        choices.append([int(x) for x in chosen])
    out["ghz_trajectories"] = {"qubits": 6, "p": 0.3, "noise_seed": 500, "choices": choices}
    # SplittableRandom(1234567).nextDouble() x 8
    out["splitmix_doubles"] = {"seed": 1234567, "values": O.uniforms(1234567, 8).tolist()}
    return out


if __name__ == "__main__":
    path = Path(__file__).resolve().parent / "goldens.json"
    path.write_text(json.dumps(compute(), indent=1) + "\n")
    print(path)
