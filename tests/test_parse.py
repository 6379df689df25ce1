"""Circuit parsers (statecraft_b200/parse.py) against the reference parser tests
(JsonCircuitParserTest.java, OpenQasmCircuitParserTest.java): each parsed circuit
is compared with the circuit the reference test builds by hand, through the naive
oracle (the reference tests' QuantumCircuit.apply), at 1e-12."""
import math

import numpy as np
import pytest

from oracle import naive
from statecraft_b200 import quantum as Q
from statecraft_b200.engine import serialize_circuit
from statecraft_b200.parse import (CircuitFormat, CircuitFormatDetector, CircuitParseException,
                                   CircuitParsers, JsonCircuitParser, OpenQasmCircuitParser)

EPS = 1e-12


def same_state(a: Q.QuantumCircuit, b: Q.QuantumCircuit) -> None:
    np.testing.assert_allclose(np.array(naive.apply(a)), np.array(naive.apply(b)), rtol=0, atol=EPS)


def bell() -> Q.QuantumCircuit:
    return Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)


# ---- JSON (JsonCircuitParserTest.java:22-121) ------------------------------------
def test_json_bell():
    c = JsonCircuitParser().parse('{"qubits": 2, "operations": ['
                                  '{"gate": "h", "target": 0}, {"gate": "cx", "control": 0, "target": 1}]}')
    same_state(c, bell())


def test_json_unknown_gate():
    with pytest.raises(CircuitParseException, match="Unknown gate"):
        JsonCircuitParser().parse('{"qubits": 1, "operations": [{"gate": "foo", "target": 0}]}')


def test_json_controlled_and_multi_control():
    src = """{"qubits": 3, "operations": [
        {"gate": "x", "target": 0}, {"gate": "x", "target": 1},
        {"gate": "ccx", "controls": [0, 1], "target": 2},
        {"gate": "mcy", "controls": [2], "target": 0},
        {"gate": "cz", "control": 2, "target": 1}]}"""
    want = (Q.QuantumCircuit(3).append(Q.PauliX(), 0).append(Q.PauliX(), 1).appendToffoli(0, 1, 2)
            .appendMultiControl(Q.PauliY(), 0, 2).appendControlledZ(2, 1))
    same_state(JsonCircuitParser().parse(src), want)


def test_json_measure_defaults_to_all_qubits():
    c = JsonCircuitParser().parse('{"qubits": 3, "operations": [{"gate": "h", "target": 0}, '
                                  '{"gate": "barrier"}, {"gate": "measure"}]}')
    assert c.operations[-1].qubits == (0, 1, 2)


def test_json_s_and_sdg():
    c = JsonCircuitParser().parse('{"qubits": 1, "operations": [{"gate": "x", "target": 0}, '
                                  '{"gate": "s", "target": 0}, {"gate": "sdg", "target": 0}]}')
    same_state(c, Q.QuantumCircuit(1).append(Q.PauliX(), 0).append(Q.SGate(), 0).append(Q.SdgGate(), 0))


@pytest.mark.parametrize("src,message", [
    ('{"qubits": 2, "operations": [{"gate": "h", "target": 0}, {"gate": "measure"}, '
     '{"gate": "x", "target": 1}]}', "cannot follow a measurement"),
    ('{"qubits": 2, "operations": [{"gate": "cx", "control": 1, "target": 1}]}', "distinct"),
    ('{"qubits": 2, "operations": [{"gate": "h", "target": 2}]}', "target qubit out of range: 2"),
    ('{"qubits": 2, "operations": [{"gate": "h", "target": 1.0}]}', "must be an integer"),
    ('{"qubits": true}', "must be an integer"),
    ('{"operations": []}', "Missing required field 'qubits'"),
    ('[1, 2]', "Root JSON value must be an object"),
    ('{"qubits": 0}', "'qubits' must be positive"),
    ('{"qubits": 3, "operations": [{"gate": "ccx", "controls": [0], "target": 2}]}',
     "exactly two control qubits"),
    ('{"qubits": 3, "operations": [{"gate": "mcx", "controls": [], "target": 2}]}', "must not be empty"),
    ('{"qubits": 3, "operations": [{"gate": "mcz", "controls": [1, 1], "target": 2}]}',
     "Duplicate measured qubit: 1"),
    ('{"qubits": 2, "operations": [{"gate": "cp", "control": 0, "target": 1}]}', "requires 'angle'"),
    ('{"qubits": 2, "operations": [{"gate": "swap", "first": 0}]}', "requires 'second'"),
])
def test_json_errors(src, message):
    with pytest.raises(CircuitParseException, match=message):
        JsonCircuitParser().parse(src)


def test_json_invalid_syntax_reports_position():
    with pytest.raises(CircuitParseException) as e:
        JsonCircuitParser().parse('{\n  "qubits": 2,\n  "operations": [ }')
    assert "Invalid JSON" in str(e.value) and e.value.line == 3


# ---- OpenQASM (OpenQasmCircuitParserTest.java:22-332) ------------------------------
def qasm(src: str) -> Q.QuantumCircuit:
    return OpenQasmCircuitParser().parse(src)


def test_qasm3_bell():
    same_state(qasm("OPENQASM 3.0;\nqubit[2] q;\n\nh q[0];\ncx q[0], q[1];\n"), bell())


def test_qasm2_bell_with_include():
    src = 'OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg qr[2];\ncreg cr[2];\n\nh qr[0];\ncx qr[0], qr[1];\n'
    same_state(qasm(src), bell())


def test_registers_flatten_in_declaration_order():
    src = "OPENQASM 3.0;\nqubit[1] ancilla;\nqubit[2] data;\n\nh data[0];\ncx data[0], ancilla[0];\n"
    same_state(qasm(src), Q.QuantumCircuit(3).append(Q.Hadamard(), 1).append(Q.CnotGate.of(), 1, 0))


def test_measurement_in_middle_rejected():
    src = "OPENQASM 3.0;\nqubit[1] q;\nbit[1] c;\n\nh q[0];\nmeasure q[0] -> c[0];\nx q[0];\n"
    with pytest.raises(CircuitParseException) as e:
        qasm(src)
    assert "measurement" in str(e.value).lower()
    assert (e.value.line, e.value.column) == (7, 1)


def test_qasm_controlled_and_multi_control():
    src = "OPENQASM 3.0;\nqubit[3] q;\n\nx q[0];\nx q[1];\nccx q[0], q[1], q[2];\ncy q[2], q[0];\ncz q[2], q[1];\n"
    want = (Q.QuantumCircuit(3).append(Q.PauliX(), 0).append(Q.PauliX(), 1).appendToffoli(0, 1, 2)
            .appendControlledY(2, 0).appendControlledZ(2, 1))
    same_state(qasm(src), want)


def test_register_wide_measurement():
    c = qasm("OPENQASM 3.0;\nqubit[3] q;\n\nh q[0];\nbarrier q;\nmeasure q;\n")
    assert c.operations[-1].qubits == (0, 1, 2)


def test_qasm2_register_wide_measurement_with_classical_target():
    c = qasm("OPENQASM 2.0;\nqreg q[2];\ncreg out[2];\n\nh q[0];\ncx q[0], q[1];\nmeasure q -> out;\n")
    assert c.operations[-1].qubits == (0, 1)


def test_qasm_s_and_sdg():
    c = qasm("OPENQASM 3.0;\nqubit[1] q;\n\nx q[0];\ns q[0];\nsdg q[0];\n")
    same_state(c, Q.QuantumCircuit(1).append(Q.PauliX(), 0).append(Q.SGate(), 0).append(Q.SdgGate(), 0))


def test_rotation_and_phase_gates():
    src = ('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[1];\n\nry((pi / 4) * 2 + pi / 2) q[0];\n'
           'p(pi / 2) q[0];\nt q[0];\ntdg q[0];\nu1(0) q[0];\n')
    s = naive.apply(qasm(src))
    assert abs(s[0]) < EPS and abs(s[1] - 1j) < EPS


def test_universal_and_rotation_gates():
    s = naive.apply(qasm("OPENQASM 3.0;\nqubit[1] q;\n\nU(pi, 0, pi) q[0];\nrx(pi) q[0];\nrz(2 * pi) q[0];\n"))
    assert abs(s[0] - 1j) < EPS and abs(s[1]) < EPS


def test_multi_control_pauli_aliases():
    src = "OPENQASM 3.0;\nqubit[3] q;\n\nx q[0];\nx q[1];\nmcy q[0], q[1], q[2];\nmcz q[0], q[1], q[2];\nmcx q[0], q[1], q[2];\n"
    want = (Q.QuantumCircuit(3).append(Q.PauliX(), 0).append(Q.PauliX(), 1)
            .appendMultiControl(Q.PauliY(), 2, 0, 1).appendMultiControl(Q.PauliZ(), 2, 0, 1)
            .appendMultiControl(Q.PauliX(), 2, 0, 1))
    same_state(qasm(src), want)


def test_bom_prefixed_qasm_directly_and_by_detection(tmp_path):
    src = "\ufeffOPENQASM 3.0;\nqubit[2] q;\n\nh q[0];\ncx q[0], q[1];\n"
    same_state(qasm(src), bell())
    path = tmp_path / "bell.qasm"
    path.write_text(src, encoding="utf-8")
    same_state(CircuitParsers.parse(path, CircuitFormat.AUTO), bell())


def test_scientific_notation_angles():
    src = "OPENQASM 3.0;\nqubit[2] q;\n\nh q[0];\nh q[1];\ncp(1e-3) q[0], q[1];\ncp(-2.5E-1) q[1], q[0];\n"
    want = (Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.Hadamard(), 1)
            .appendControlledPhase(1e-3, 0, 1).appendControlledPhase(-2.5e-1, 1, 0))
    same_state(qasm(src), want)


@pytest.mark.parametrize("src,message", [
    ("OPENQASM 2.0;\nqreg q[1];\ngate custom a { x a; }\ncustom q[0];\n", "Unsupported OpenQASM construct"),
    ("OPENQASM 2.0;\nqreg q[1];\ncreg c[1];\nif (c==1) x q[0];\n", "Unsupported OpenQASM construct"),
    ("OPENQASM 2.0;\nqreg q[2];\ncreg c[1];\nmeasure q -> c;\n", "Measurement source and target sizes must match"),
    ("OPENQASM 3.0;\nqubit[1] q;\nrz(pi / 0) q[0];\n", "division by zero"),
    ("OPENQASM 4.0;\nqubit[1] q;\n", "Only OPENQASM 2.0 and 3.0"),
    ("OPENQASM 3.0;\nh q[0];\n", "Unknown qubit register"),
    ("OPENQASM 3.0;\nqubit[2] q;\ncx q[0], q[0];\n", "CNOT control and target must be distinct"),
    ("OPENQASM 3.0;\nqubit[2] q;\nh q[2];\n", "Qubit index out of range: 2"),
    ("OPENQASM 3.0;\nqubit[2] q;\nh q;\n", "Expected indexed qubit operand"),
    ("OPENQASM 3.0;\nqubit[2] q;\nrx q[0];\n", "expects 1 parameter"),
    ("OPENQASM 3.0;\nqubit[3] q;\nmcx q[0], q[0], q[2];\n", "Duplicate control qubit: 0"),
    ("OPENQASM 3.0;\nqubit[2] q;\nh q[0];\nqubit[1] r;\n", "Register declarations must appear before"),
    ("OPENQASM 3.0;\nqubit[2] q;\nqubit[1] q;\n", "Duplicate register declaration"),
    ("OPENQASM 3.0;\nqubit[0] q;\n", "Register size must be positive"),
    ("OPENQASM 3.0;\n", "Missing qubit register declaration"),
    ("OPENQASM 3.0;\nqubit[1] q;\n/* open\n", "Unterminated block comment"),
    ("OPENQASM 3.0;\nqubit[1] q;\nfoo q[0];\n", "Unsupported instruction: foo"),
    ("OPENQASM 3.0;\nqubit[1] q;\nh q[0] $\n", "Unexpected character"),
])
def test_qasm_errors(src, message):
    with pytest.raises(CircuitParseException, match=message):
        qasm(src)


def test_qasm_error_position():
    with pytest.raises(CircuitParseException) as e:
        qasm("OPENQASM 3.0;\nqubit[1] q;\n  rz(pi / 0) q[0];\n")
    assert (e.value.line, e.value.column) == (3, 9)


def test_comments_u2_identity_and_aliases():
    src = ("// header\nOPENQASM 2.0; /* block */\nqreg a[2];\nu2(0, pi) a[0]; // = H\n"
           "id a[1];\ncnot a[0], a[1];\ncu1(pi/3) a[1], a[0];\nswap a[0], a[1];\n")
    want = (Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
            .appendControlledPhase(math.pi / 3, 1, 0).appendSwap(0, 1))
    same_state(qasm(src), want)


def test_format_detection(tmp_path):
    assert CircuitFormat.fromOption(" QASM ") == CircuitFormat.QASM
    with pytest.raises(ValueError):
        CircuitFormat.fromOption("yaml")
    assert CircuitFormatDetector.detectByExtension("x.qasm3") == CircuitFormat.QASM
    assert CircuitFormatDetector.detectByExtension("x.JSON") == CircuitFormat.JSON
    assert CircuitFormatDetector.detectByContent("  // c\n/* d */ OPENQASM 3.0;") == CircuitFormat.QASM
    assert CircuitFormatDetector.detectByContent('{"qubits": 1}') is None
    path = tmp_path / "circuit.txt"
    path.write_text('{"qubits": 2, "operations": [{"gate": "h", "target": 0}, '
                    '{"gate": "cx", "control": 0, "target": 1}]}')
    with pytest.raises(CircuitParseException, match="Unable to detect circuit format"):
        CircuitParsers.parse(path)
    same_state(CircuitParsers.parse(path, CircuitFormat.JSON), bell())


def test_parsed_circuit_serializes_like_the_built_one():
    # the device op stream of a parsed circuit is the stream of the same circuit
    # built through the API
    src = "OPENQASM 3.0;\nqubit[3] q;\nh q[0];\nrx(0.25) q[1];\nccx q[0], q[1], q[2];\ncp(0.5) q[2], q[0];\n"
    want = (Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.rx(0.25), 1).appendToffoli(0, 1, 2)
            .appendControlledPhase(0.5, 2, 0))
    a, na = serialize_circuit(qasm(src))
    b, nb = serialize_circuit(want)
    import ctypes
    assert na == nb and ctypes.string_at(a, ctypes.sizeof(a)) == ctypes.string_at(b, ctypes.sizeof(b))
