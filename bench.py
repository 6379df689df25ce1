#!/usr/bin/env python3
"""Benchmark of the B200 statevector engine on its headline workload.

Workload (one step): 30-qubit complex128 brick-wall circuit of depth 40 (U3 on every
qubit, CNOT brick, a 29-control multi-controlled Z on the all-ones pattern and an
RZZ(gamma) on a seeded random pair per layer; angles from SplitMix64 seed 3030),
run from |0...0> with fusion, followed by countsAll(8192) with seed 42.
Metric: gate-level amplitude updates per second (1.643e12 per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (one process per GPU under torchrun, weak
scaling); the state vector of one circuit does not shard without an exchange.
`--impl reference` times the CPU restatement of the reference engine (the Java
engine cannot run here: no JDK) on a bounded sample of the same 30-qubit workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "amp-updates/s (30q c128 brick-wall depth 40 + MCZ29 + RZZ, fused, countsAll 8192)"
UNIT = "amp-updates/s"


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=40)
    ap.add_argument("--shots", type=int, default=8192)
    ap.add_argument("--tile-qubits", type=int, default=0)
    ap.add_argument("--sweep-budget", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=["statevector", "c1", "qaoa", "adjoint", "trajectories",
                                           "blocks"],
                    default="statevector",
                    help="statevector: the headline line; c1: the 20-qubit plain drop-in; "
                         "the others time the batched QAOA, adjoint-gradient and "
                         "noisy-trajectory workloads (one JSON line each, 1 GPU)")
    ap.add_argument("--instances", type=int, default=4096, help="QAOA batch size")
    ap.add_argument("--trajectories", type=int, default=1024, help="trajectory batch size")
    ap.add_argument("--channel", choices=["depolarizing", "amplitude_damping"],
                    default="depolarizing", help="trajectories: noise channel")
    ap.add_argument("--autotune", action="store_true", help="trajectories: time tile shapes")
    ap.add_argument("--no-tune", action="store_true", help="QAOA: fixed kernel shape")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    try:
                        rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
                    except ValueError:
                        pass
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        load = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in load),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(r[2] for r in rows)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def ncu_traffic() -> dict:
    """DRAM bytes per sweep launch from the committed ncu summary, when present."""
    p = ROOT / "profiles" / "sweep_kernel_traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


# ---------------------------------------------------------------------------
# CPU baseline (the oracle restatement of the reference engine, OpenMP)
# ---------------------------------------------------------------------------
_NATIVE_ORACLE = None


def native_oracle():
    """The oracle's C restatement built with -O3 -march=native for the host that runs
    the bench (compiled here, into a temporary directory, because the library in
    oracle/_build is built -O2 for any x86-64); same -ffp-contract=off arithmetic."""
    global _NATIVE_ORACLE
    if _NATIVE_ORACLE is None:
        import ctypes

        from statecraft_b200 import _abi as A

        out = Path(tempfile.mkdtemp(prefix="sc_oracle_native_")) / "libsc_oracle_native.so"
        cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
        subprocess.run([cc, "-O3", "-march=native", "-ffp-contract=off", "-fno-fast-math",
                        "-fPIC", "-fopenmp", "-std=c11", "-shared", "-o", str(out),
                        str(ROOT / "oracle" / "sc_oracle.c"), "-lm"], check=True)
        lib = ctypes.CDLL(str(out))
        lib.scx_apply_op.restype = ctypes.c_int
        lib.scx_apply_op.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                     ctypes.POINTER(A.ScOp), ctypes.POINTER(ctypes.c_double),
                                     ctypes.c_int64]
        _NATIVE_ORACLE = lib
    return _NATIVE_ORACLE


class CpuSample:
    """A bounded CPU sample of the headline workload: the first `n_ops` operations of
    the 30-qubit brick-wall generator (seed 3030, MCZ + RZZ), applied one full-state
    pass each by the oracle's restatement of the reference engine's per-gate loops
    (StatevectorOps.java), on one pre-touched 16 GiB state reused between samples."""

    def __init__(self, qubits: int = 30, n_ops: int = 47):
        import ctypes

        from statecraft_b200 import quantum as Q
        from statecraft_b200 import workloads as W
        from statecraft_b200.engine import serialize_circuit

        self.qubits = qubits
        c = W.brickwall_circuit(qubits, 1, seed=3030, mcz=True, rzz=True)
        self.circuit = Q.QuantumCircuit(qubits, tuple(c.operations[:n_ops]))
        self.ops, self.n_ops = serialize_circuit(self.circuit)
        self.updates = W.amp_updates(self.circuit)
        self.state = np.zeros(2 << qubits)
        self.state[0] = 1.0
        self.state[1::4096] = 0.0  # touch every page once before timing
        self.lib = native_oracle()
        self._dp = self.state.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self.cores = len(os.sched_getaffinity(0))

    def run(self) -> float:
        """Seconds for one pass over the sample's operations."""
        import ctypes

        from statecraft_b200 import _abi as A

        base = ctypes.addressof(self.ops)
        t0 = time.perf_counter()
        for i in range(self.n_ops):
            op = ctypes.cast(base + i * ctypes.sizeof(A.ScOp), ctypes.POINTER(A.ScOp))
            rc = self.lib.scx_apply_op(self._dp, self.qubits, op, None, 0)
            assert rc == 0
        return time.perf_counter() - t0

    def describe(self) -> str:
        return (f"C restatement of StatevectorEngine's per-gate loops (OpenMP {self.cores} threads, "
                f"gcc -O3 -march=native -ffp-contract=off) on the first {self.n_ops} operations "
                f"of the same {self.qubits}-qubit brick-wall generator (layer 0: U3 on every "
                f"qubit, CNOT brick, MCZ, RZZ); the Java engine is unavailable on this host (no JDK)")


def cpu_baseline() -> dict:
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    s = CpuSample()
    s.run()  # warm-up pass
    dt = s.run()
    out = {"value": s.updates / dt, "unit": UNIT, "cores": s.cores, "kind": "port",
           "seconds": dt, "sample": s.describe()}
    del s
    return out


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    # each step: the first 10 operations of the 30-qubit workload (a few seconds on 16 cores)
    s = CpuSample(n_ops=10)
    for _ in range(args.warmup):
        s.run()
    secs = [s.run() for _ in range(args.steps)]
    value = s.updates * args.steps / sum(secs)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(secs) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"brick-wall U3+CNOT+MCZ+RZZ, {s.qubits} qubits, first "
                                   f"{s.n_ops} operations per step (bounded CPU sample of the "
                                   f"30q x 40 workload)",
                       "qubits": s.qubits, "ops_per_step": s.n_ops},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": s.cores, "kind": "port",
                             "sample": s.describe()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# secondary workloads (one GPU; one JSON line each)
# ---------------------------------------------------------------------------
def _timed(fn, steps: int, warmup: int):
    import torch

    for _ in range(max(warmup, 0)):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        out = fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / steps, out


def run_qaoa(args) -> dict:
    """4096 QAOA ring instances, n ~ U{10..22}, p = 4, one captured graph per evaluation."""
    from statecraft_b200 import _abi as A
    from statecraft_b200 import workloads as W
    from statecraft_b200.batch import QaoaRingBatch
    from statecraft_b200.engine import B200Config, NativeContext

    count = args.instances
    b = W.qaoa_instances(count, 4, 4096)
    ctx = NativeContext(B200Config())
    res = {}
    for name, dt in (("c128", A.SC_C128), ("c64", A.SC_C64)):
        q = QaoaRingBatch(b.n_qubits, b.gammas, b.betas, dtype=dt, tune=not args.no_tune,
                          context=ctx)
        sec, e = _timed(q.evaluate, args.steps, args.warmup)
        info = q.info()
        res[name] = {"s_per_batch": sec, "energies": e, "info": info,
                     "hbm_gbs": info["hbm_bytes_per_run"] / sec / 1e9}
        q.close()
    ctx.close()
    upd = QaoaRingBatch.amp_updates(b.n_qubits, 4)
    err = np.abs(res["c64"]["energies"] - res["c128"]["energies"])
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    sec = res["c128"]["s_per_batch"]
    return {"metric": f"amp-updates/s (batched QAOA ring ansatz, {count} instances, n ~ U{{10..22}}, "
                      "p = 4, <sum ZZ> per instance, c128)",
            "value": upd / sec, "unit": "amp-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "qaoa-ring batch", "instances": count, "layers": 4,
                       "n_range": [10, 22], "seed": 4096, "amp_updates_per_step": upd},
            "instances_per_s": count / sec,
            "c128": {k: v for k, v in res["c128"].items() if k != "energies"},
            "c64": {k: v for k, v in res["c64"].items() if k != "energies"},
            "c64_energy_error_vs_c128": {"max": float(err.max()), "mean": float(err.mean())},
            "roofline": {"bound": "hbm", "achieved": res["c128"]["hbm_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": res["c128"]["hbm_gbs"] / peak, "traffic": None}}


def run_adjoint(args) -> dict:
    """26-qubit hardware-efficient ansatz, 624 angles, 64-term Pauli sum: adjoint
    gradients against central finite differences on the plain (forward) engine."""
    from statecraft_b200 import _abi as A
    from statecraft_b200 import workloads as W
    from statecraft_b200.adjoint import AdjointEngine
    from statecraft_b200.engine import B200Config

    n, layers, h = 26, 12, 1e-6
    ops, n_ops, n_params = W.hea_ops(n, layers)
    theta = W.hea_params(n_params, 2626)
    x, z, c = W.random_pauli_sum(n, 64, 6464)
    out = {}
    for name, dt in (("c128", A.SC_C128), ("c64", A.SC_C64)):
        eng = AdjointEngine(B200Config(dtype=dt))
        sec, (e, g) = _timed(lambda: eng.value_and_grad(n, ops, n_ops, theta, x, z, c),
                             args.steps, args.warmup)
        out[name] = {"s_per_gradient": sec, "value": e, "grad": g}
        eng.close()
    # finite differences on the plain engine: the same circuit with the angles baked in
    eng = AdjointEngine(B200Config())
    idx = np.linspace(0, n_params - 1, 8).astype(int)
    fd = []
    t_eval = []
    for k in idx:
        vals = []
        for sgn in (1, -1):
            th = theta.copy()
            th[k] += sgn * h
            t0 = time.perf_counter()
            vals.append(eng.expectation(n, ops, n_ops, th, x, z, c))
            t_eval.append(time.perf_counter() - t0)
        fd.append((vals[0] - vals[1]) / (2 * h))
    eng.close()
    fd = np.array(fd)
    s_eval = float(np.median(t_eval))
    fd_s = 2 * n_params * s_eval
    g128 = out["c128"]["grad"]
    diff = np.abs(g128[idx] - fd)
    fd_noise = 4 * np.finfo(float).eps * float(np.sum(np.abs(c))) * n_ops / h
    sec = out["c128"]["s_per_gradient"]
    return {"metric": "adjoint gradients/s (26q c128 hardware-efficient ansatz, 12 layers, "
                      "624 angles, 64-term Pauli sum) vs central finite differences",
            "value": 1.0 / sec, "unit": "gradients/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "adjoint HEA", "qubits": n, "layers": layers,
                       "angles": n_params, "terms": 64, "angle_seed": 2626, "h_seed": 6464},
            "energy": out["c128"]["value"],
            "finite_differences": {"h": h, "s_per_evaluation": s_eval,
                                   "evaluations_per_gradient": 2 * n_params,
                                   "gradients_per_s": 1.0 / fd_s,
                                   "checked_angles": idx.tolist()},
            "speedup_vs_fd": fd_s / sec,
            "max_abs_diff_vs_fd": float(diff.max()), "fd_noise_bound": fd_noise,
            "c64": {"gradients_per_s": 1.0 / out["c64"]["s_per_gradient"],
                    "max_abs_grad_error_vs_c128": float(np.abs(out["c64"]["grad"] - g128).max()),
                    "energy_error_vs_c128": abs(out["c64"]["value"] - out["c128"]["value"])}}


def run_trajectories_bench(args) -> dict:
    """Noisy 22-qubit GHZ, a single-qubit channel after every gate on each touched
    qubit, 1024 complex64 trajectories per batch, countsAll(64) each.  The default
    channel is depolarizing p = 1e-3 (a Pauli mixture: branches drawn on the host,
    applied inside the fused sweeps); ``--channel amplitude_damping`` uses amplitude
    damping gamma = 1e-3 (state-dependent weights, each record weighed, drawn and
    applied on the device).  ``value`` times whole batches through ``run_trajectories``
    (the captured graph of the batch after the first call; outcomes and choices copied
    back every step); ``kernel_stats`` and the roofline come from one more batch on a
    context timing each kernel class."""
    from statecraft_b200 import _abi as A
    from statecraft_b200 import noise as N
    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import B200Config, NativeContext
    from statecraft_b200.trajectories import run_trajectories, touched_qubit_depolarizing

    n, traj, shots, p = 22, args.trajectories, 64, 1e-3
    c = W.ghz_circuit(n)
    if args.channel == "amplitude_damping":
        kraus = tuple(np.array(k.matrix, dtype=complex).reshape(2, 2)
                      for k in N.AmplitudeDampingChannel(p, (0,)).krausDecomposition())
        rec = [N.FlatChannel(i, q, kraus) for i, op in enumerate(c.operations)
               for q in sorted(op.qubits_touched())]
    else:
        rec = touched_qubit_depolarizing(c, p)
    ctx = NativeContext(B200Config(dtype=A.SC_C64, autotune=args.autotune))
    sec, r = _timed(lambda: run_trajectories(c, rec, traj, 2024, shots, 4096, context=ctx),
                    args.steps, args.warmup)
    info = ctx.trajectories_info()
    launches = {k: v["launches"] for k, v in ctx.kernel_stats().items() if v["launches"]}
    plan = ctx.plan_stats()
    ctx.close()
    tctx = NativeContext(B200Config(dtype=A.SC_C64, timing=True, tile_qubits=info["tile_qubits"]))
    run_trajectories(c, rec, traj, 2024, shots, 4096, context=tctx)
    stats = {k: v for k, v in tctx.kernel_stats().items() if v["launches"]}
    tctx.close()
    sw = stats.get("sweep", {"ms": 0.0, "bytes": 0.0, "launches": 0})
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    gbs = sw["bytes"] / (sw["ms"] / 1e3) / 1e9 if sw["ms"] else None
    h = r.histogram()
    ghz = (h.get(0, 0) + h.get((1 << n) - 1, 0)) / (traj * shots)
    chan = "amplitude damping gamma" if args.channel == "amplitude_damping" else "depolarizing p"
    steps_launched = args.steps + args.warmup
    return {"metric": f"trajectories/s (noisy GHZ 22q c64, touched-qubit {chan}=1e-3, "
                      f"{traj} trajectories x countsAll(64))",
            "value": traj / sec, "unit": "trajectories/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "noisy GHZ trajectories", "qubits": n, "trajectories": traj,
                       "shots": shots, "channel": args.channel, "p": p, "noise_seed": 2024,
                       "measure_seed": 4096, "noise_records": len(rec),
                       "sweeps": plan["sweeps"], "stages": plan["stages"],
                       "tile_qubits": info["tile_qubits"], "nr": info["nr"],
                       "graph": info["graph"], "autotune_ms": info["tuned_ms"]},
            "gpu_launches": sum(launches.values()) // max(1, steps_launched),
            "kernel_stats": stats,
            "ghz_fraction": ghz,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": (gbs / peak) if gbs else None, "traffic": None}}


def run_c1(args) -> dict:
    """The 20-qubit plain drop-in: brick-wall U3 + CNOT, 20 layers, angles from
    SplittableRandom(2020), |0..0> start, final state and countsAll(1024) with seed 42.
    `value` times sc_run + sc_sample on the device (state resident); `e2e` times
    StatevectorB200Engine.simulate with the final state (16 MiB) and the histogram
    copied back.  The 16 MiB state fits in L2; a 512 MiB buffer is written between
    timed steps so every step starts with L2 holding other data."""
    import torch

    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import (B200Config, MeasurementInstruction, NativeContext,
                                        SimulationRequest, StatevectorB200Engine,
                                        serialize_circuit)

    n, layers, shots = 20, 20, 1024
    circuit = W.brickwall_circuit(n, layers, seed=2020)
    ops, n_ops = serialize_circuit(circuit)
    updates = W.amp_updates(circuit)
    qubits = list(range(n))
    steps = max(args.steps, 1) * 50
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    ctx = NativeContext(B200Config(timing=True))
    stream = torch.cuda.ExternalStream(ctx.lib.sc_stream(ctx.handle))

    def step():
        ctx.run_ops(n, ops, n_ops)
        return ctx.sample(qubits, shots, 42)

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.reset_kernel_stats()
    total_ms = 0.0
    with ClockSampler(0) as clk:
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            total_ms += a.elapsed_time(b)
    stats = ctx.kernel_stats()
    plan = ctx.plan_stats()
    ctx.close()
    launches = sum(v["launches"] for v in stats.values())
    engine = StatevectorB200Engine(B200Config())
    req = SimulationRequest.zeroState(circuit).withMeasurement(
        MeasurementInstruction.countsAll(shots).withSeed(42), True)
    engine.simulate(req)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        res = engine.simulate(req)
    e2e_s = (time.perf_counter() - t0) / steps
    assert sum(res.measurement.counts.values()) == shots
    engine.close()
    ms = total_ms / steps
    sw = stats.get("sweep", {"launches": 0, "ms": 0.0, "bytes": 0.0})
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    gbs = (sw["bytes"] / (sw["ms"] / 1e3) / 1e9) if sw["ms"] else None
    return {"metric": "amp-updates/s (20q c128 brick-wall depth 20, final state + countsAll 1024)",
            "value": updates / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "brick-wall U3+CNOT, 20 qubits x 20 layers, countsAll(1024) "
                                   "seed 42, final state, c128", "qubits": n, "layers": layers,
                       "angle_seed": 2020, "shots": shots, "amp_updates_per_step": updates,
                       "sweeps_per_step": plan["sweeps"], "stages_per_step": plan["stages"],
                       "l2": "state (16 MiB) fits in L2; a 512 MiB write between timed steps"},
            "gpu_launches": launches // steps,
            "kernel_stats": stats,
            "e2e": {"value": updates / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n_ops * 280,
                    "d2h_bytes_per_step": (16 << n) + 4 * shots, "seconds_per_step": e2e_s},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": (gbs / peak) if gbs else None, "traffic": None,
                         "note": "sweeps of an L2-resident state: bytes per sweep over its time"},
            "clocks": clk.summary()}


def run_blocks(args) -> dict:
    """Dense tensor-core blocks against the sweep path on a circuit made for them:
    28 qubits, 60 rounds of 12 gates inside random 5-qubit windows (dense random
    two-qubit unitaries, CNOTs, U3, controlled phases; a 27-control MCZ every third
    round).  Both timings are sc_run on the device with the state resident."""
    import torch

    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import B200Config, NativeContext, serialize_circuit

    n = 28
    c = W.dense_window_circuit(n, 60, seed=2828)
    ops, n_ops = serialize_circuit(c)
    updates = W.amp_updates(c)
    out = {}
    for name, thr in (("sweeps", "0"), ("blocks", "1"), ("blocks_cost64", "64")):
        os.environ["STATECRAFT_B200_DENSE_BLOCKS"] = thr
        ctx = NativeContext(B200Config(timing=True))
        for _ in range(max(args.warmup, 1)):
            ctx.run_ops(n, ops, n_ops)
        ctx.reset_kernel_stats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ctx.run_ops(n, ops, n_ops)
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / args.steps
        stats = {k: v for k, v in ctx.kernel_stats().items() if v["launches"]}
        out[name] = {"s_per_run": sec, "plan": ctx.plan_stats(), "kernel_stats": stats}
        ctx.close()
    os.environ.pop("STATECRAFT_B200_DENSE_BLOCKS", None)
    blk = out["blocks"]["kernel_stats"].get("block", {"launches": 0, "ms": 0.0, "bytes": 0.0})
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    gbs = blk["bytes"] / (blk["ms"] / 1e3) / 1e9 if blk["ms"] else None
    return {"metric": "amp-updates/s (28q dense 5-qubit-window circuit, tensor-core blocks vs sweeps)",
            "value": updates / out["blocks"]["s_per_run"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * out["blocks"]["s_per_run"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "dense 5-qubit windows", "qubits": n, "rounds": 60,
                       "seed": 2828, "amp_updates_per_step": updates},
            "sweeps_only": {"value": updates / out["sweeps"]["s_per_run"],
                            "ms_per_step": 1e3 * out["sweeps"]["s_per_run"],
                            "plan": out["sweeps"]["plan"]},
            "blocks": {"plan": out["blocks"]["plan"], "kernel_stats": out["blocks"]["kernel_stats"],
                       "note": "every run of gates on <= 5 qubits (at least 3) as a dense block"},
            "blocks_cost64": {"value": updates / out["blocks_cost64"]["s_per_run"],
                              "ms_per_step": 1e3 * out["blocks_cost64"]["s_per_run"],
                              "plan": out["blocks_cost64"]["plan"]},
            "roofline_block_kernel": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                      "frac": (gbs / peak) if gbs else None}}


# ---------------------------------------------------------------------------
# the B200 engine
# ---------------------------------------------------------------------------
def main(argv=None) -> int:
    args = parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return 0
    if args.workload != "statevector":
        fn = {"c1": run_c1, "qaoa": run_qaoa, "adjoint": run_adjoint,
              "trajectories": run_trajectories_bench, "blocks": run_blocks}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return 0

    import torch
    import torch.distributed as dist

    from statecraft_b200 import _abi as A
    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import (B200Config, MeasurementInstruction, NativeContext,
                                        SimulationRequest, StatevectorB200Engine,
                                        serialize_circuit)

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))

    n, layers, shots = args.qubits, args.layers, args.shots
    circuit = W.brickwall_circuit(n, layers, seed=3030, mcz=True, rzz=True)
    ops, n_ops = serialize_circuit(circuit)
    updates = W.amp_updates(circuit)
    qubits = list(range(n))
    cfg = B200Config(device=local_rank, timing=True, tile_qubits=args.tile_qubits,
                     sweep_budget=args.sweep_budget)
    ctx = NativeContext(cfg)
    stream = torch.cuda.ExternalStream(ctx.lib.sc_stream(ctx.handle), device=local_rank)

    def step():
        ctx.run_ops(n, ops, n_ops)
        return ctx.sample(qubits, shots, 42)

    for _ in range(max(args.warmup, 0)):
        step()
    ctx.reset_kernel_stats()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        start.record(stream)
        for _ in range(args.steps):
            outcomes = step()
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    dev_ms = start.elapsed_time(end)
    stats = ctx.kernel_stats()
    plan = ctx.plan_stats()
    t = torch.tensor([dev_ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    max_ms = float(t.item())
    value = world * updates * args.steps / (max_ms / 1e3)
    launches = sum(v["launches"] for v in stats.values())
    ctx.close()

    # e2e through the public engine API: host circuit in, host histogram out
    e2e = None
    if not args.no_e2e:
        engine = StatevectorB200Engine(B200Config(device=local_rank, tile_qubits=args.tile_qubits,
                                                  sweep_budget=args.sweep_budget))
        req = SimulationRequest.zeroState(circuit).withMeasurement(
            MeasurementInstruction.countsAll(shots).withSeed(42), False)
        engine.simulate(req)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = engine.simulate(req)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        te = torch.tensor([e2e_s], device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_s = float(te.item())
        assert sum(res.measurement.counts.values()) == shots
        e2e = {"value": world * updates * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": n_ops * 280, "d2h_bytes_per_step": shots * 4,
               "seconds_per_step": e2e_s / args.steps}
        engine.close()

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    sw = stats.get("sweep", {"launches": 0, "ms": 0.0, "bytes": 0.0})
    roofline = None
    if sw["launches"] > 0 and sw["ms"] > 0:
        per_launch_bytes = sw["bytes"] / sw["launches"]
        avg_s = sw["ms"] / sw["launches"] / 1e3
        achieved = per_launch_bytes / avg_s / 1e9
        peak = hbm if hbm else 6650.0
        tr = ncu_traffic()
        traffic = None
        if tr.get("bytes_per_amplitude"):
            traffic = tr["bytes_per_amplitude"] * (2 ** n)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "peak_source": "measured" if hbm else "fallback",
                    "kernel": "k_sweep (fused tile sweep)",
                    "algorithmic_bytes_per_launch": per_launch_bytes,
                    "avg_launch_ms": sw["ms"] / sw["launches"],
                    "share_of_step": sw["ms"] / max(dev_ms, 1e-9)}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"brick-wall U3+CNOT+MCZ{n - 1}+RZZ, {n} qubits x {layers} layers, "
                                   f"countsAll({shots}) seed 42, c128",
                       "qubits": n, "layers": layers, "shots": shots, "angle_seed": 3030,
                       "replicas": world,
                       "l2": f"state {2 ** n * 16 / 2 ** 30:.0f} GiB per GPU exceeds the 126 MB L2",
                       "amp_updates_per_step": updates,
                       "sweeps_per_step": plan["sweeps"], "gates_per_step": plan["gates"],
                       "stages_per_step": plan["stages"]},
            "gpu_launches": launches,
            "kernel_stats": stats,
            "roofline": roofline,
            "e2e": e2e,
            "clocks": clk.summary()}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
