"""Parsed circuits on the GPU engine: OpenQASM and JSON sources using every gate the
parsers accept run through StatevectorB200Engine and match the oracle (1e-12)."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200.engine import (B200Config, MeasurementInstruction, SimulationRequest,
                                    StatevectorB200Engine, serialize_circuit)
from statecraft_b200.parse import JsonCircuitParser, OpenQasmCircuitParser

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = StatevectorB200Engine(B200Config())
    yield e
    e.close()


def qasm_program(n: int, gates: int, seed: int) -> str:
    rng = np.random.default_rng(seed)
    lines = ["OPENQASM 3.0;", f"qubit[{n - 2}] q;", "qubit[2] anc;", "bit[%d] c;" % n]
    def qb(k):
        return f"q[{k}]" if k < n - 2 else f"anc[{k - n + 2}]"
    def angle():
        return f"{rng.uniform(-3, 3):.6f} * pi / 3"
    for _ in range(gates):
        kind = rng.integers(0, 12)
        qs = [int(x) for x in rng.permutation(n)[:4]]
        if kind == 0:
            g = ["h", "x", "y", "z", "s", "sdg", "t", "tdg", "id"][rng.integers(0, 9)]
            lines.append(f"{g} {qb(qs[0])};")
        elif kind == 1:
            g = ["p", "u1", "rx", "ry", "rz"][rng.integers(0, 5)]
            lines.append(f"{g}({angle()}) {qb(qs[0])};")
        elif kind == 2:
            lines.append(f"U({angle()}, {angle()}, {angle()}) {qb(qs[0])};")
        elif kind == 3:
            lines.append(f"u3({angle()}, {angle()}, {angle()}) {qb(qs[0])};")
        elif kind == 4:
            lines.append(f"u2({angle()}, {angle()}) {qb(qs[0])};")
        elif kind in (5, 6):
            g = ["cx", "cnot", "cy", "cz"][rng.integers(0, 4)]
            lines.append(f"{g} {qb(qs[0])}, {qb(qs[1])};")
        elif kind == 7:
            lines.append(f"ccx {qb(qs[0])}, {qb(qs[1])}, {qb(qs[2])};")
        elif kind == 8:
            g = ["mcx", "mcy", "mcz"][rng.integers(0, 3)]
            k = int(rng.integers(2, 5))
            lines.append(f"{g} " + ", ".join(qb(x) for x in qs[:k]) + ";")
        elif kind == 9:
            lines.append(f"swap {qb(qs[0])}, {qb(qs[1])};")
        elif kind == 10:
            g = ["cp", "cu1"][rng.integers(0, 2)]
            lines.append(f"{g}({angle()}) {qb(qs[0])}, {qb(qs[1])};")
        else:
            lines.append("barrier q, anc;")
    return "\n".join(lines) + "\n"


def oracle_state(circuit):
    ops, n_ops = serialize_circuit(circuit)
    st = O.initial_state(circuit.qubitCount)
    rc, _ = O.run(circuit.qubitCount, ops, n_ops, st)
    assert rc == 0
    return st


@pytest.mark.parametrize("n,seed", [(6, 1), (14, 2), (20, 3)])
def test_parsed_qasm_matches_oracle(engine, n, seed):
    c = OpenQasmCircuitParser().parse(qasm_program(n, 300, seed))
    got = engine.simulate(SimulationRequest.zeroState(c)).finalState.data()
    np.testing.assert_allclose(got, oracle_state(c), rtol=0, atol=1e-12)


def test_parsed_qasm_with_measurement(engine):
    c = OpenQasmCircuitParser().parse(qasm_program(12, 120, 9) + "measure q;\nmeasure anc;\n")
    res = engine.simulate(SimulationRequest.zeroState(c)
                          .withMeasurement(MeasurementInstruction.countsAll(512).withSeed(7), True))
    assert sum(res.measurement.counts.values()) == 512
    np.testing.assert_allclose(res.finalState.data(), oracle_state(c), rtol=0, atol=1e-12)


def test_parsed_json_matches_oracle(engine):
    rng = np.random.default_rng(5)
    n, ops = 10, []
    for _ in range(200):
        q = [int(x) for x in rng.permutation(n)[:3]]
        k = rng.integers(0, 6)
        if k == 0:
            ops.append({"gate": ["h", "x", "y", "z", "s", "sdg"][rng.integers(0, 6)], "target": q[0]})
        elif k == 1:
            ops.append({"gate": ["cx", "cy", "cz"][rng.integers(0, 3)], "control": q[0], "target": q[1]})
        elif k == 2:
            ops.append({"gate": "cp", "control": q[0], "target": q[1], "angle": float(rng.uniform(0, 6))})
        elif k == 3:
            ops.append({"gate": "swap", "first": q[0], "second": q[1]})
        elif k == 4:
            ops.append({"gate": "ccx", "controls": q[:2], "target": q[2]})
        else:
            ops.append({"gate": ["mcx", "mcy", "mcz"][rng.integers(0, 3)], "controls": q[:2],
                        "target": q[2]})
    c = JsonCircuitParser().parse(json.dumps({"qubits": n, "operations": ops}))
    got = engine.simulate(SimulationRequest.zeroState(c)).finalState.data()
    np.testing.assert_allclose(got, oracle_state(c), rtol=0, atol=1e-12)
