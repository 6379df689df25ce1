"""External-comparison runner on the B200 engine.

Command-line twin of StateCraft's ``StatecraftComparisonRunner``
(``engines/src/test/java/com/omaarr90/statecraft/engines/comparison/StatecraftComparisonRunner.java:26-282``),
the runner its benchmark harness (``scripts/benchmark/comparison/run_comparison.py``)
starts once per fixture.  Same arguments, same run protocol, same one-line JSON
result, so the harness can start this module in place of the Java runner:

    python -m statecraft_b200.comparison --fixture-id bell --category ideal \\
        --circuit-json bell.statecraft.json --warmup-runs 1 --timed-runs 5

- The circuit is read with the JSON circuit parser.
- Noiseless fixtures: ``warmup-runs`` untimed and ``timed-runs`` timed runs of
  ``simulate(zeroState(circuit))``; each timed run is wall-clock time around the
  call (device upload, kernels and the final-state read-back included, like the
  reference's ``System.nanoTime`` bracket).  The result carries the probabilities
  and the amplitudes of the last run.
- Noisy fixtures: the noise model is ``afterAllGates(channel(q))`` for each noise
  qubit; a timed run averages the probabilities of ``noise-trajectories`` runs with
  noise seeds ``noise-seed + t`` (the reference's convention, ``:70-86``).
- Numbers are printed like Java's ``String.format(Locale.US, "%.17g", x)``.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from decimal import Decimal
from typing import Callable, Optional, Sequence

import numpy as np

from . import noise as N
from . import quantum as Q
from .parse import CircuitFormat, CircuitParsers

RUNNER_NAME = "statecraft"
DEFAULT_NOISE_SEED = 0x51A7EC0FFEEA


def _int_list(value: str) -> list[int]:
    return [] if not value.strip() else [int(v.strip()) for v in value.split(",")]


def parse_options(argv: Sequence[str]) -> argparse.Namespace:
    """Options.parse (StatecraftComparisonRunner.java:218-264)."""
    ap = argparse.ArgumentParser(prog="python -m statecraft_b200.comparison", add_help=False)
    ap.add_argument("--fixture-id", default="")
    ap.add_argument("--category", default="")
    ap.add_argument("--circuit-json", required=True)
    ap.add_argument("--warmup-runs", type=int, default=1)
    ap.add_argument("--timed-runs", type=int, default=5)
    ap.add_argument("--parallelism", type=int, default=1)
    ap.add_argument("--noise-type", default=None)
    ap.add_argument("--noise-qubits", type=_int_list, default=[])
    ap.add_argument("--noise-trajectories", type=int, default=512)
    ap.add_argument("--noise-seed", type=int, default=DEFAULT_NOISE_SEED)
    ap.add_argument("--noise-probability", type=float, default=0.0)
    ap.add_argument("--noise-gamma", type=float, default=0.0)
    ap.add_argument("--noise-lambda", type=float, default=0.0)
    ap.add_argument("--noise-t1", type=float, default=0.0)
    ap.add_argument("--noise-t2", type=float, default=0.0)
    ap.add_argument("--noise-gate-time", type=float, default=0.0)
    opts = ap.parse_args(list(argv))
    if opts.noise_type is not None and not opts.noise_qubits:
        ap.error("--noise-qubits is required when --noise-type is provided")
    return opts


def noise_model(opts: argparse.Namespace) -> Optional[N.NoiseModel]:
    """buildNoiseModel / createChannel (StatecraftComparisonRunner.java:88-107)."""
    if opts.noise_type is None:
        return None
    make = {
        "depolarizing": lambda q: N.ErrorChannel.depolarizing(opts.noise_probability, q),
        "phase_flip": lambda q: N.ErrorChannel.phaseFlip(opts.noise_probability, q),
        "amplitude_damping": lambda q: N.ErrorChannel.amplitudeDamping(opts.noise_gamma, q),
        "phase_damping": lambda q: N.ErrorChannel.phaseDamping(opts.noise_lambda, q),
        "thermal_relaxation": lambda q: N.ErrorChannel.thermalRelaxation(
            opts.noise_t1, opts.noise_t2, opts.noise_gate_time, q),
    }.get(opts.noise_type)
    if make is None:
        raise ValueError(f"unknown noise type: {opts.noise_type}")
    builder = N.NoiseModel.builder()
    for q in opts.noise_qubits:
        builder.afterAllGates(make(q))
    return builder.build()


def _probabilities(state: Q.StateVector) -> np.ndarray:
    d = np.asarray(state.data(), dtype=np.float64)
    return d[0::2] * d[0::2] + d[1::2] * d[1::2]


def run_fixture(opts: argparse.Namespace, engine, request_type) -> dict:
    """main (StatecraftComparisonRunner.java:30-57): returns the result fields."""
    circuit = CircuitParsers.parse(opts.circuit_json, CircuitFormat.JSON)
    model = noise_model(opts)

    def run_once(seed: int) -> Q.StateVector:
        req = request_type.zeroState(circuit)
        if model is not None:
            req = req.withNoiseModel(model).withNoiseSeed(seed)
        return engine.simulate(req).finalState

    for i in range(opts.warmup_runs):
        run_once(opts.noise_seed + i)
    timed: list[float] = []
    final = None
    if model is None:
        for i in range(opts.timed_runs):
            t0 = time.perf_counter_ns()
            final = run_once(opts.noise_seed + i)
            timed.append((time.perf_counter_ns() - t0) / 1e6)
        probs = _probabilities(final) if final is not None else np.zeros(0)
    else:
        probs = np.zeros(1 << circuit.qubitCount)
        for _ in range(opts.timed_runs):
            t0 = time.perf_counter_ns()
            agg = np.zeros(1 << circuit.qubitCount)
            for t in range(opts.noise_trajectories):
                agg += _probabilities(run_once(opts.noise_seed + t))
            probs = agg * (1.0 / opts.noise_trajectories)
            timed.append((time.perf_counter_ns() - t0) / 1e6)
    n_ops = sum(1 for op in circuit.operations if not isinstance(op, Q.MeasureOperation))
    result = {
        "runner": RUNNER_NAME, "fixture_id": opts.fixture_id, "category": opts.category,
        "status": "ok", "qubits": circuit.qubitCount, "operations": n_ops,
        "threads": opts.parallelism, "warmup_runs": opts.warmup_runs,
        "timed_runs": opts.timed_runs,
        "noise_trajectories": 0 if model is None else opts.noise_trajectories,
        "timed_runs_ms": timed, "mean_ms": float(np.mean(timed)) if timed else 0.0,
        "probabilities": probs,
    }
    if final is not None:
        result["statevector"] = np.asarray(final.data(), dtype=np.float64)
    return result


def java_g17(x: float) -> str:
    """String.format(Locale.US, "%.17g", x): Java pads the shortest round-trip digits
    of x (those of Double.toString) with zeros to 17 significant digits, and writes
    magnitudes in [1e-4, 1e17) in fixed notation, others as d.ddd...e+XX."""
    x = float(x)
    if x != x:
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    sign = "-" if math.copysign(1.0, x) < 0 else ""
    if x == 0.0:
        return sign + "0." + "0" * 16
    _, digits, exp = Decimal(repr(abs(x))).as_tuple()
    e10 = len(digits) + exp - 1  # decimal exponent of the leading digit
    ds = "".join(map(str, digits)).ljust(17, "0")[:17]
    if -4 <= e10 < 17:
        if e10 >= 0:
            whole, frac = ds[:e10 + 1], ds[e10 + 1:]
            return sign + whole + ("." + frac if frac else "")
        return sign + "0." + "0" * (-e10 - 1) + ds
    return f"{sign}{ds[0]}.{ds[1:]}e{'-' if e10 < 0 else '+'}{abs(e10):02d}"


def render(result: dict) -> str:
    """renderResult (StatecraftComparisonRunner.java:117-140): field order and number
    format of the reference's result line."""
    def s(v: str) -> str:
        return json.dumps(v, ensure_ascii=False)

    def arr(values) -> str:
        return "[" + ",".join(java_g17(v) for v in values) + "]"

    parts = [f'"runner":{s(result["runner"])}', f'"fixture_id":{s(result["fixture_id"])}',
             f'"category":{s(result["category"])}', f'"status":{s(result["status"])}',
             f'"qubits":{result["qubits"]}', f'"operations":{result["operations"]}',
             f'"threads":{result["threads"]}', f'"warmup_runs":{result["warmup_runs"]}',
             f'"timed_runs":{result["timed_runs"]}',
             f'"noise_trajectories":{result["noise_trajectories"]}',
             f'"timed_runs_ms":{arr(result["timed_runs_ms"])}',
             f'"mean_ms":{java_g17(result["mean_ms"])}',
             f'"probabilities":{arr(result["probabilities"])}']
    if "statevector" in result:
        d = result["statevector"]
        parts.append('"statevector":[' + ",".join(
            f"[{java_g17(d[2 * k])},{java_g17(d[2 * k + 1])}]" for k in range(len(d) // 2)) + "]")
    return "{" + ",".join(parts) + "}"


def main(argv: Optional[Sequence[str]] = None,
         engine_factory: Optional[Callable[[], object]] = None) -> int:
    from .engine import B200Config, SimulationRequest, StatevectorB200Engine

    opts = parse_options(sys.argv[1:] if argv is None else argv)
    engine = engine_factory() if engine_factory else StatevectorB200Engine(B200Config())
    try:
        print(render(run_fixture(opts, engine, SimulationRequest)), flush=True)
    finally:
        close = getattr(engine, "close", None)
        if close:
            close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
