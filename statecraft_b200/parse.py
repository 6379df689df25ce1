"""Circuit parsers: JSON and OpenQASM 2.0 / 3.0 source -> ``QuantumCircuit``.

Host-side mirror of StateCraft's parsing package
(``core/src/main/java/com/omaarr90/statecraft/core/parse/``): the same input
formats, gate names, defaults and error rules, so a circuit file that the
reference CLI accepts builds the same ``QuantumCircuit`` here, and the engine's
``serialize_circuit`` turns it into the device op stream.

- ``JsonCircuitParser`` follows ``JsonCircuitParser.java:26-386``: a root object
  with an integer ``qubits`` and an optional ``operations`` array of objects with a
  ``gate`` name and the fields ``target``, ``control``, ``first``, ``second``,
  ``angle``, ``qubits`` and ``controls``.
- ``OpenQasmCircuitParser`` follows ``OpenQasmCircuitParser.java:28-970``: version
  2.0 or 3.0, ``include``, ``qreg``/``creg`` and ``qubit``/``bit`` declarations
  (registers flatten in declaration order), the standard single-qubit gates with
  constant angle expressions (numbers, ``pi``, + - * / and parentheses),
  ``cx``/``cy``/``cz``/``ccx``/``mcx``/``mcy``/``mcz``/``swap``/``cp``/``cu1``,
  ``barrier`` and ``measure``; user gate definitions and classical control flow
  are rejected.
- ``CircuitFormat`` / ``CircuitFormatDetector`` / ``CircuitParsers`` follow
  ``CircuitFormat.java``, ``CircuitFormatDetector.java:20-79`` and
  ``CircuitParsers.java:18-52`` (by extension, then by an ``OPENQASM`` header).

Errors raise ``CircuitParseException`` with the reference's messages and, where
the reference reports one, a 1-based line and column.
"""
from __future__ import annotations

import enum
import json
import math
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

from . import quantum as Q

__all__ = ["CircuitParseException", "CircuitFormat", "CircuitFormatDetector", "CircuitParsers",
           "JsonCircuitParser", "OpenQasmCircuitParser"]


class CircuitParseException(ValueError):
    """CircuitParseException.java:7-43: message plus an optional 1-based position."""

    def __init__(self, message: str, line: int = 0, column: int = 0):
        super().__init__(message)
        self.line = line if line > 0 else None
        self.column = column if column > 0 else None


def _strip_bom(source: str) -> str:
    return source[1:] if source.startswith("\ufeff") else source


# ---------------------------------------------------------------------------
# JSON
# ---------------------------------------------------------------------------

def _is_int(value) -> bool:
    return isinstance(value, int) and not isinstance(value, bool)


def _is_number(value) -> bool:
    return isinstance(value, (int, float)) and not isinstance(value, bool)


class JsonCircuitParser:
    """JsonCircuitParser.java:26-386."""

    def parse(self, source: str) -> Q.QuantumCircuit:
        if source is None:
            raise TypeError("source")
        qubits, ops = self._definition(_strip_bom(source))
        return self._build(qubits, ops)

    # -- reading ------------------------------------------------------------
    @staticmethod
    def _definition(source: str):
        try:
            root = json.loads(source)
        except json.JSONDecodeError as e:
            raise CircuitParseException(f"Invalid JSON: {e.msg}", e.lineno, e.colno) from e
        if root is None:
            raise CircuitParseException("JSON source is empty")
        if not isinstance(root, dict):
            raise CircuitParseException("Root JSON value must be an object")
        qubits = JsonCircuitParser._required_int(root, "qubits", "root")
        ops = []
        node = root.get("operations")
        if node is not None:
            if not isinstance(node, list):
                raise CircuitParseException("'operations' must be an array")
            for index, op in enumerate(node):
                if not isinstance(op, dict):
                    raise CircuitParseException(f"operations[{index}] must be an object")
                ctx = f"operations[{index}]"
                gate = op.get("gate")
                if gate is None:
                    raise CircuitParseException(f"Missing required field 'gate' in {ctx}")
                if not isinstance(gate, str):
                    raise CircuitParseException(f"Field 'gate' in {ctx} must be a string")
                spec = {"gate": gate}
                for field in ("target", "control", "first", "second"):
                    spec[field] = JsonCircuitParser._optional_int(op, field, ctx)
                angle = op.get("angle")
                if angle is not None and not _is_number(angle):
                    raise CircuitParseException(f"Field 'angle' in {ctx} must be a number")
                spec["angle"] = None if angle is None else float(angle)
                for field in ("qubits", "controls"):
                    spec[field] = JsonCircuitParser._optional_int_list(op, field, ctx)
                ops.append(spec)
        return qubits, ops

    @staticmethod
    def _required_int(node: dict, field: str, ctx: str) -> int:
        value = node.get(field)
        if value is None:
            raise CircuitParseException(f"Missing required field '{field}' in {ctx}")
        if not _is_int(value):
            raise CircuitParseException(f"Field '{field}' in {ctx} must be an integer")
        return value

    @staticmethod
    def _optional_int(node: dict, field: str, ctx: str) -> Optional[int]:
        value = node.get(field)
        if value is None:
            return None
        if not _is_int(value):
            raise CircuitParseException(f"Field '{field}' in {ctx} must be an integer")
        return value

    @staticmethod
    def _optional_int_list(node: dict, field: str, ctx: str) -> Optional[list]:
        value = node.get(field)
        if value is None:
            return None
        if not isinstance(value, list):
            raise CircuitParseException(f"Field '{field}' in {ctx} must be an array")
        for element in value:
            if not _is_int(element):
                raise CircuitParseException(f"Field '{field}' in {ctx} must contain integers")
        return list(value)

    # -- building -----------------------------------------------------------
    @staticmethod
    def _need(value, message: str):
        if value is None:
            raise CircuitParseException(message)
        return value

    @staticmethod
    def _index(index: int, n: int, label: str) -> None:
        if index < 0 or index >= n:
            raise CircuitParseException(f"{label} qubit out of range: {index}")

    @staticmethod
    def _sorted_qubits(qubits: list, n: int) -> list:
        if not qubits:
            raise CircuitParseException("Measurement qubit list must not be empty")
        for q in qubits:
            if q < 0 or q >= n:
                raise CircuitParseException(f"Measured qubit out of range: {q}")
        out = sorted(qubits)
        for a, b in zip(out, out[1:]):
            if a == b:
                raise CircuitParseException(f"Duplicate measured qubit: {b}")
        return out

    @staticmethod
    def _controls(controls, n: int, missing: str) -> list:
        if controls is None:
            raise CircuitParseException(missing)
        if not controls:
            raise CircuitParseException("control qubit list must not be empty")
        return JsonCircuitParser._sorted_qubits(controls, n)

    def _build(self, n: int, ops: list) -> Q.QuantumCircuit:
        if n <= 0:
            raise CircuitParseException("'qubits' must be positive")
        c = Q.QuantumCircuit(n)
        measured = False
        single = {"h": Q.Hadamard, "x": Q.PauliX, "y": Q.PauliY, "z": Q.PauliZ, "s": Q.SGate,
                  "sdg": Q.SdgGate}
        multi = {"mcx": Q.PauliX, "mcy": Q.PauliY, "mcz": Q.PauliZ}
        need, index = self._need, self._index
        for op in ops:
            gate = op["gate"].strip().lower()
            if measured and gate not in ("measure", "barrier"):
                raise CircuitParseException(
                    f"Unitary gate '{gate}' cannot follow a measurement operation")
            if gate in single:
                t = need(op["target"], f"gate '{gate}' requires 'target'")
                index(t, n, "target")
                c = c.append(single[gate](), t)
            elif gate in ("cx", "cy", "cz"):
                ctl = need(op["control"], f"gate '{gate}' requires 'control'")
                t = need(op["target"], f"gate '{gate}' requires 'target'")
                if gate != "cx" and ctl == t:
                    raise CircuitParseException(
                        f"gate '{gate}' requires distinct control and target qubits")
                index(ctl, n, "control")
                index(t, n, "target")
                if gate == "cx":
                    if ctl == t:
                        raise CircuitParseException(
                            "gate 'cx' requires distinct control and target qubits")
                    c = c.append(Q.CnotGate.of(), ctl, t)
                elif gate == "cy":
                    c = c.appendControlledY(ctl, t)
                else:
                    c = c.appendControlledZ(ctl, t)
            elif gate == "swap":
                a = need(op["first"], "gate 'swap' requires 'first'")
                b = need(op["second"], "gate 'swap' requires 'second'")
                index(a, n, "first")
                index(b, n, "second")
                if a == b:
                    raise CircuitParseException("gate 'swap' requires distinct qubits")
                c = c.appendSwap(a, b)
            elif gate == "cp":
                ctl = need(op["control"], "gate 'cp' requires 'control'")
                t = need(op["target"], "gate 'cp' requires 'target'")
                angle = need(op["angle"], "gate 'cp' requires 'angle'")
                if not math.isfinite(angle):
                    raise CircuitParseException("gate 'cp' requires a finite angle")
                index(ctl, n, "control")
                index(t, n, "target")
                if ctl == t:
                    raise CircuitParseException(
                        "gate 'cp' requires distinct control and target qubits")
                c = c.appendControlledPhase(angle, ctl, t)
            elif gate == "ccx":
                t = need(op["target"], "gate 'ccx' requires 'target'")
                cs = self._controls(op["controls"], n,
                                    "gate 'ccx' requires 'controls' with exactly two qubits")
                if len(cs) != 2:
                    raise CircuitParseException("gate 'ccx' requires exactly two control qubits")
                if t in cs:
                    raise CircuitParseException("gate 'ccx' requires distinct controls and target")
                index(t, n, "target")
                c = c.appendToffoli(cs[0], cs[1], t)
            elif gate in multi:
                t = need(op["target"], f"gate '{gate}' requires 'target'")
                cs = self._controls(op["controls"], n, f"gate '{gate}' requires 'controls'")
                if t in cs:
                    raise CircuitParseException(
                        f"gate '{gate}' requires distinct controls and target")
                index(t, n, "target")
                c = c.appendMultiControl(multi[gate](), t, *cs)
            elif gate == "measure":
                measured = True
                qs = op["qubits"] if op["qubits"] is not None else list(range(n))
                c = c.measure(*self._sorted_qubits(qs, n))
            elif gate == "barrier":
                pass  # no simulation effect
            else:
                raise CircuitParseException(f"Unknown gate: '{op['gate']}'")
        return c


# ---------------------------------------------------------------------------
# OpenQASM 2.0 / 3.0
# ---------------------------------------------------------------------------

_IDENT, _NUMBER, _STRING, _SYMBOL, _EOF = "identifier", "number", "string", "symbol", "eof"
_SYMBOL_CHARS = set(";,[]()/-+*")


@dataclass(frozen=True)
class _Token:
    kind: str
    text: str
    line: int
    column: int


class _Tokenizer:
    """Lazy tokenizer: a token is read only when the parser asks for it, so an
    unsupported construct is reported before characters past it are examined."""

    def __init__(self, source: str):
        self.s = source
        self.i = 0
        self.line = 1
        self.column = 1

    def _advance(self) -> None:
        ch = self.s[self.i]
        self.i += 1
        if ch == "\n":
            self.line += 1
            self.column = 1
        else:
            self.column += 1

    def _skip_trivia(self) -> None:
        s, n = self.s, len(self.s)
        while self.i < n:
            if s[self.i].isspace():
                self._advance()
            elif s.startswith("//", self.i):
                while self.i < n and s[self.i] != "\n":
                    self._advance()
            elif s.startswith("/*", self.i):
                self._advance()
                self._advance()
                while self.i + 1 < n and not s.startswith("*/", self.i):
                    self._advance()
                if self.i + 1 >= n:
                    raise CircuitParseException("Unterminated block comment", self.line, self.column)
                self._advance()
                self._advance()
            else:
                return

    def next(self) -> _Token:
        self._skip_trivia()
        s, n = self.s, len(self.s)
        if self.i >= n:
            return _Token(_EOF, "", self.line, self.column)
        line, col, start = self.line, self.column, self.i
        ch = s[self.i]
        if ch.isalpha() or ch == "_":
            while self.i < n and (s[self.i].isalnum() or s[self.i] == "_"):
                self._advance()
            return _Token(_IDENT, s[start:self.i], line, col)
        if ch.isdigit() or (ch == "." and self.i + 1 < n and s[self.i + 1].isdigit()):
            return _Token(_NUMBER, self._number(), line, col)
        if ch == '"':
            return _Token(_STRING, self._string(line, col), line, col)
        if s.startswith("->", self.i):
            self._advance()
            self._advance()
            return _Token(_SYMBOL, "->", line, col)
        if ch in _SYMBOL_CHARS:
            self._advance()
            return _Token(_SYMBOL, ch, line, col)
        raise CircuitParseException(f"Unexpected character: '{ch}'", line, col)

    def _number(self) -> str:
        s, n, start = self.s, len(self.s), self.i
        dot = exp = False
        while self.i < n:
            ch = s[self.i]
            if ch.isdigit():
                self._advance()
            elif ch == "." and not dot and not exp:
                dot = True
                self._advance()
            elif ch in "eE" and not exp:
                k = self.i + 1
                if k < n and s[k] in "+-":
                    k += 1
                if k < n and s[k].isdigit():
                    exp = True
                    self._advance()
                    if s[self.i] in "+-":
                        self._advance()
                else:
                    break
            else:
                break
        return s[start:self.i]

    def _string(self, line: int, col: int) -> str:
        s, n = self.s, len(self.s)
        self._advance()
        out = []
        while self.i < n:
            ch = s[self.i]
            if ch == '"':
                self._advance()
                return "".join(out)
            if ch == "\\":
                self._advance()
                if self.i >= n:
                    break
            out.append(s[self.i])
            self._advance()
        raise CircuitParseException("Unterminated string literal", line, col)


@dataclass(frozen=True)
class _Register:
    size: int
    offset: int


_UNSUPPORTED = {"gate", "opaque", "if", "reset", "def", "defcal", "for", "while", "box", "delay",
                "cal", "let", "const"}


def _phase_gate(name: str, angle: float) -> Q.MatrixSingleQubitGate:
    return Q.MatrixSingleQubitGate(name, 1, 0, 0, complex(math.cos(angle), math.sin(angle)))


def _u_gate(name: str, theta: float, phi: float, lam: float) -> Q.MatrixSingleQubitGate:
    g = Q.u3(theta, phi, lam)
    return Q.MatrixSingleQubitGate(name, *(g.element(r, c) for r in (0, 1) for c in (0, 1)))


class _QasmParser:
    def __init__(self, source: str):
        self.tok = _Tokenizer(source)
        self.cur = self.tok.next()
        self.qregs: dict[str, _Register] = {}
        self.cregs: dict[str, _Register] = {}
        self.nq = 0
        self.nc = 0

    # -- token helpers ------------------------------------------------------
    def _adv(self) -> None:
        self.cur = self.tok.next()

    def _err(self, message: str, tok: Optional[_Token] = None) -> CircuitParseException:
        t = tok or self.cur
        return CircuitParseException(message, t.line, t.column)

    def _expect(self, kind: str, message: str) -> _Token:
        if self.cur.kind != kind:
            raise self._err(message)
        t = self.cur
        self._adv()
        return t

    def _expect_ident(self, word: str) -> _Token:
        t = self._expect(_IDENT, "Expected identifier")
        if t.text != word:
            raise self._err(f"Expected '{word}'", t)
        return t

    def _is_ident(self, word: str) -> bool:
        return self.cur.kind == _IDENT and self.cur.text == word

    def _is_sym(self, sym: str) -> bool:
        return self.cur.kind == _SYMBOL and self.cur.text == sym

    def _match(self, sym: str) -> bool:
        if self._is_sym(sym):
            self._adv()
            return True
        return False

    def _expect_sym(self, sym: str) -> None:
        if not self._is_sym(sym):
            raise self._err(f"Expected '{sym}'")
        self._adv()

    def _integer(self, t: _Token) -> int:
        if any(ch in t.text for ch in ".eE"):
            raise self._err(f"Expected integer but got '{t.text}'", t)
        return int(t.text)

    def _double(self, t: _Token) -> float:
        try:
            value = float(t.text)
        except ValueError as e:
            raise self._err(f"Invalid number: {t.text}", t) from e
        if not math.isfinite(value):
            raise self._err(f"Invalid finite number: {t.text}", t)
        return value

    # -- program ------------------------------------------------------------
    def program(self):
        self._expect_ident("OPENQASM")
        vt = self._expect(_NUMBER, "Expected OpenQASM version number")
        version = self._double(vt)
        if abs(version - 2.0) > 1e-9 and abs(version - 3.0) > 1e-9:
            raise self._err("Only OPENQASM 2.0 and 3.0 are supported", vt)
        self._expect_sym(";")
        instructions = []
        started = False
        while self.cur.kind != _EOF:
            if self._is_ident("include"):
                self._adv()
                self._expect(_STRING, "Expected include file name")
                self._expect_sym(";")
                continue
            decl = {"qreg": ("q", True), "creg": ("c", True), "qubit": ("q", False),
                    "bit": ("c", False)}.get(self.cur.text if self.cur.kind == _IDENT else "")
            if decl is not None:
                if started:
                    raise self._err("Register declarations must appear before instructions")
                self._declaration(*decl)
                continue
            started = True
            instructions.append(self._instruction())
        if not self.qregs:
            raise CircuitParseException("Missing qubit register declaration")
        return self.nq, instructions

    def _declaration(self, kind: str, legacy: bool) -> None:
        kw = self.cur
        self._adv()
        if legacy:  # qreg name[size];
            name = self._expect(_IDENT, "Expected register name")
            self._expect_sym("[")
            st = self._expect(_NUMBER, "Expected register size")
            size = self._integer(st)
            self._expect_sym("]")
        else:  # qubit[size] name;  (size 1 without brackets)
            size, st = 1, kw
            if self._match("["):
                st = self._expect(_NUMBER, "Expected register size")
                size = self._integer(st)
                self._expect_sym("]")
            name = self._expect(_IDENT, "Expected register name")
        self._expect_sym(";")
        if size <= 0:
            raise self._err("Register size must be positive", st)
        regs = self.qregs if kind == "q" else self.cregs
        if name.text in regs:
            raise self._err(f"Duplicate register declaration: {name.text}", kw)
        if kind == "q":
            regs[name.text] = _Register(size, self.nq)
            self.nq += size
        else:
            regs[name.text] = _Register(size, self.nc)
            self.nc += size

    def _instruction(self):
        gt = self._expect(_IDENT, "Expected instruction")
        gate = gt.text.lower()
        loc = (gt.line, gt.column)
        if gate == "barrier":
            self._operand(self.qregs, "qubit", True)
            while self._match(","):
                self._operand(self.qregs, "qubit", True)
            self._expect_sym(";")
            return ("barrier", loc)
        if gate == "measure":
            qubits = self._operand(self.qregs, "qubit", True)
            if self._match("->"):
                bits = self._operand(self.cregs, "bit", True)
                if len(bits) != len(qubits):
                    raise CircuitParseException("Measurement source and target sizes must match", *loc)
            self._expect_sym(";")
            return ("measure", loc, qubits)
        if gate in _UNSUPPORTED:
            raise self._err(f"Unsupported OpenQASM construct: {gt.text}", gt)
        params = self._parameters()
        qubits = [self._operand(self.qregs, "qubit", False)[0]]
        while self._match(","):
            qubits.append(self._operand(self.qregs, "qubit", False)[0])
        self._expect_sym(";")
        return self._gate(gate, params, qubits, loc)

    def _operand(self, regs: dict, label: str, wide: bool) -> list:
        rt = self._expect(_IDENT, f"Expected {label} register")
        reg = regs.get(rt.text)
        if reg is None:
            raise self._err(f"Unknown {label} register: {rt.text}", rt)
        if self._match("["):
            it = self._expect(_NUMBER, f"Expected {label} index")
            index = self._integer(it)
            self._expect_sym("]")
            if index < 0 or index >= reg.size:
                raise self._err(f"{label.capitalize()} index out of range: {index}", it)
            return [reg.offset + index]
        if not wide:
            raise self._err(f"Expected indexed {label} operand", rt)
        return list(range(reg.offset, reg.offset + reg.size))

    def _parameters(self) -> list:
        if not self._match("("):
            return []
        params = []
        if not self._is_sym(")"):
            while True:
                value = self._additive()
                if not math.isfinite(value):
                    raise self._err("Angle expression must be finite")
                params.append(value)
                if not self._match(","):
                    break
        self._expect_sym(")")
        return params

    def _additive(self) -> float:
        value = self._multiplicative()
        while True:
            if self._match("+"):
                value += self._multiplicative()
            elif self._match("-"):
                value -= self._multiplicative()
            else:
                return value

    def _multiplicative(self) -> float:
        value = self._unary()
        while True:
            if self._match("*"):
                value *= self._unary()
            elif self._is_sym("/"):
                op = self.cur
                self._adv()
                divisor = self._unary()
                if divisor == 0.0:
                    raise self._err("Angle expression division by zero", op)
                value /= divisor
            else:
                return value

    def _unary(self) -> float:
        if self._match("+"):
            return self._unary()
        if self._match("-"):
            return -self._unary()
        if self.cur.kind == _NUMBER:
            t = self.cur
            self._adv()
            return self._double(t)
        if self._is_ident("pi"):
            self._adv()
            return math.pi
        if self._match("("):
            value = self._additive()
            self._expect_sym(")")
            return value
        raise self._err("Expected angle expression")

    def _gate(self, gate: str, params: list, qubits: list, loc):
        def counts(n_params: int, n_qubits: Optional[int]) -> None:
            if len(params) != n_params:
                raise CircuitParseException(
                    f"Gate '{gate}' expects {n_params} parameter(s), got {len(params)}", *loc)
            if n_qubits is not None and len(qubits) != n_qubits:
                raise CircuitParseException(
                    f"Gate '{gate}' expects {n_qubits} qubit operand(s), got {len(qubits)}", *loc)

        fixed = {"h": Q.Hadamard, "x": Q.PauliX, "y": Q.PauliY, "z": Q.PauliZ, "s": Q.SGate,
                 "sdg": Q.SdgGate}
        if gate in fixed:
            counts(0, 1)
            return ("single", loc, fixed[gate](), qubits[0])
        if gate in ("t", "tdg"):
            counts(0, 1)
            name, angle = ("T", math.pi / 4.0) if gate == "t" else ("Tdg", -math.pi / 4.0)
            return ("single", loc, _phase_gate(name, angle), qubits[0])
        if gate in ("id", "iden"):
            counts(0, 1)
            return ("noop", loc, qubits[0])
        if gate in ("p", "u1", "rx", "ry", "rz"):
            counts(1, 1)
            a = params[0]
            g = {"rx": Q.rx, "ry": Q.ry, "rz": Q.rz}.get(gate)
            return ("single", loc, g(a) if g else _phase_gate(gate, a), qubits[0])
        if gate in ("u", "u3"):
            counts(3, 1)
            return ("single", loc, _u_gate("U" if gate == "u" else "u3", *params), qubits[0])
        if gate == "u2":
            counts(2, 1)
            return ("single", loc, _u_gate("u2", math.pi / 2.0, *params), qubits[0])
        if gate in ("cx", "cnot"):
            counts(0, 2)
            return ("cnot", loc, qubits[0], qubits[1])
        if gate in ("cy", "cz"):
            counts(0, 2)
            return ("controlled", loc, gate[1], qubits[0], qubits[1])
        if gate == "ccx":
            counts(0, 3)
            return ("multi", loc, "x", qubits[:2], qubits[2])
        if gate in ("mcx", "mcy", "mcz"):
            counts(0, None)
            if len(qubits) < 2:
                raise CircuitParseException(f"Gate '{gate}' requires controls and a target", *loc)
            return ("multi", loc, gate[2], qubits[:-1], qubits[-1])
        if gate == "swap":
            counts(0, 2)
            return ("swap", loc, qubits[0], qubits[1])
        if gate in ("cp", "cu1"):
            counts(1, 2)
            return ("cphase", loc, params[0], qubits[0], qubits[1])
        raise CircuitParseException(f"Unsupported instruction: {gate}", *loc)


class OpenQasmCircuitParser:
    """OpenQasmCircuitParser.java:28-970."""

    def parse(self, source: str) -> Q.QuantumCircuit:
        if source is None:
            raise TypeError("source")
        n, instructions = _QasmParser(_strip_bom(source)).program()
        return self._build(n, instructions)

    @staticmethod
    def _build(n: int, instructions: list) -> Q.QuantumCircuit:
        if n <= 0:
            raise CircuitParseException("qubit register size must be positive")

        def index(q: int, loc) -> None:
            if q < 0 or q >= n:
                raise CircuitParseException(f"Qubit index out of range: {q}", *loc)

        def pair(a: int, b: int, label: str, loc) -> None:
            index(a, loc)
            index(b, loc)
            if a == b:
                raise CircuitParseException(f"{label} must be distinct", *loc)

        paulis = {"x": Q.PauliX, "y": Q.PauliY, "z": Q.PauliZ}
        c = Q.QuantumCircuit(n)
        measured = False
        for ins in instructions:
            kind, loc = ins[0], ins[1]
            if kind == "barrier":
                continue
            if kind == "measure":
                measured = True
                for q in ins[2]:
                    index(q, loc)
                c = c.measure(*ins[2])
                continue
            if measured:
                raise CircuitParseException("Unitary gate cannot follow a measurement operation", *loc)
            if kind == "single":
                index(ins[3], loc)
                c = c.append(ins[2], ins[3])
            elif kind == "noop":
                index(ins[2], loc)
            elif kind == "cnot":
                pair(ins[2], ins[3], "CNOT control and target", loc)
                c = c.append(Q.CnotGate.of(), ins[2], ins[3])
            elif kind == "controlled":
                pair(ins[3], ins[4], "Controlled gate qubits", loc)
                c = (c.appendControlledY if ins[2] == "y" else c.appendControlledZ)(ins[3], ins[4])
            elif kind == "multi":
                controls, target = ins[3], ins[4]
                if not controls:
                    raise CircuitParseException("Multi-control gate requires at least one control", *loc)
                index(target, loc)
                prev = None
                for ctl in sorted(controls):
                    index(ctl, loc)
                    if ctl == target:
                        raise CircuitParseException("Control and target must be distinct", *loc)
                    if ctl == prev:
                        raise CircuitParseException(f"Duplicate control qubit: {ctl}", *loc)
                    prev = ctl
                c = c.appendMultiControl(paulis[ins[2]](), target, *controls)
            elif kind == "swap":
                pair(ins[2], ins[3], "SWAP qubits", loc)
                c = c.appendSwap(ins[2], ins[3])
            elif kind == "cphase":
                pair(ins[3], ins[4], "Controlled-phase qubits", loc)
                c = c.appendControlledPhase(ins[2], ins[3], ins[4])
        return c


# ---------------------------------------------------------------------------
# format selection
# ---------------------------------------------------------------------------

class CircuitFormat(enum.Enum):
    """CircuitFormat.java: json, qasm or auto (detect)."""

    JSON = "json"
    QASM = "qasm"
    AUTO = "auto"

    @staticmethod
    def fromOption(value: str) -> "CircuitFormat":
        normalized = value.strip().lower()
        for f in CircuitFormat:
            if f.value == normalized:
                return f
        raise ValueError(f"Unsupported format: {value}")


class CircuitFormatDetector:
    """CircuitFormatDetector.java:20-79: by file extension, then by an OPENQASM header
    after whitespace, comments and a byte-order mark."""

    @staticmethod
    def detect(path, source: str) -> CircuitFormat:
        by_ext = CircuitFormatDetector.detectByExtension(path)
        if by_ext is not None:
            return by_ext
        by_content = CircuitFormatDetector.detectByContent(source)
        if by_content is not None:
            return by_content
        raise CircuitParseException(
            "Unable to detect circuit format; specify --format qasm or --format json.")

    @staticmethod
    def detectByExtension(path) -> Optional[CircuitFormat]:
        name = Path(path).name.lower()
        if name.endswith(".qasm") or name.endswith(".qasm3"):
            return CircuitFormat.QASM
        if name.endswith(".json"):
            return CircuitFormat.JSON
        return None

    @staticmethod
    def detectByContent(source: str) -> Optional[CircuitFormat]:
        i, n = 0, len(source)
        while i < n:
            ch = source[i]
            if ch == "\ufeff" or ch.isspace():
                i += 1
            elif source.startswith("//", i):
                while i < n and source[i] != "\n":
                    i += 1
            elif source.startswith("/*", i):
                end = source.find("*/", i + 2)
                i = n if end < 0 else end + 2
            else:
                break
        return CircuitFormat.QASM if source.startswith("OPENQASM", i) else None


class CircuitParsers:
    """CircuitParsers.java:18-52."""

    @staticmethod
    def selectParser(fmt: CircuitFormat, path, source: str):
        resolved = CircuitFormatDetector.detect(path, source) if fmt == CircuitFormat.AUTO else fmt
        return JsonCircuitParser() if resolved == CircuitFormat.JSON else OpenQasmCircuitParser()

    @staticmethod
    def parse(path, fmt: CircuitFormat = CircuitFormat.AUTO) -> Q.QuantumCircuit:
        try:
            source = _strip_bom(Path(path).read_text(encoding="utf-8"))
        except OSError as e:
            raise CircuitParseException(f"Failed to read circuit file: {path}") from e
        return CircuitParsers.selectParser(fmt, path, source).parse(source)
