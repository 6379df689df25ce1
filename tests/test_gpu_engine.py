"""GPU parity tests: the B200 engine through the C ABI against the CPU oracle.

Bar: complex128 amplitudes within 1e-12 max-abs of the oracle (the reference
tests' EPS); seeded counts identical when both sides consume the same uniforms,
except draws within 1e-12 of a CDF boundary (counted, must be rare); complex64
within 2e-5 max-abs; Pauli expectations within 1e-12; adjoint gradients within
1e-8 of parameter-shift.
"""
import math

import numpy as np
import pytest

import randcirc as RCirc
import refcircuits as RC
from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import quantum as Q
from statecraft_b200 import workloads as W
from statecraft_b200.engine import (B200Config, MeasurementInstruction, NativeContext,
                                    SimulationRequest, StatevectorB200Engine, serialize_circuit)
from statecraft_b200.noise import ErrorChannel, NoiseModel

pytestmark = pytest.mark.gpu

EPS = 1e-12


@pytest.fixture(scope="module")
def fused():
    e = StatevectorB200Engine(B200Config(fusion=True))
    yield e
    e.close()


@pytest.fixture(scope="module")
def unfused():
    e = StatevectorB200Engine(B200Config(fusion=False))
    yield e
    e.close()


@pytest.fixture(scope="module")
def c64():
    e = StatevectorB200Engine(B200Config(dtype=A.SC_C64))
    yield e
    e.close()


def _oracle_state(c, init=None):
    ops, n_ops = serialize_circuit(c)
    st = O.initial_state(c.qubitCount, init)
    rc, _ = O.run(c.qubitCount, ops, n_ops, st)
    assert rc == 0
    return st


# ---- the reference's own engine tests -----------------------------------------
@pytest.mark.parametrize("name", [c[0] for c in RC.cases()])
@pytest.mark.parametrize("mode", ["fused", "unfused"])
def test_reference_cases(name, mode, fused, unfused):
    _, request, expected = {c[0]: c for c in RC.cases()}[name]
    engine = fused if mode == "fused" else unfused
    st = engine.simulate(request).finalState.data()
    np.testing.assert_allclose(st, RC.to_interleaved(expected), rtol=0, atol=EPS)


def test_22_qubit_basis_kat(fused):
    request, idx = RC.large_basis_case()
    st = fused.simulate(request).finalState
    assert st.real(idx) == pytest.approx(1.0, abs=EPS)
    assert st.imag(idx) == pytest.approx(0.0, abs=EPS)
    assert float(np.sum(st.data() ** 2)) == pytest.approx(1.0, abs=1e-10)


def test_rejects_above_dense_limit():
    e = StatevectorB200Engine(B200Config(max_qubits=29))
    with pytest.raises(A.UnsupportedOperationException, match="supports up to 29 qubits"):
        e.simulate(SimulationRequest.zeroState(Q.QuantumCircuit(30)))
    e.close()


def test_unitary_after_measurement_throws(fused):
    c = Q.QuantumCircuit(1).append(Q.Hadamard(), 0).measure(0).append(Q.PauliX(), 0)
    req = SimulationRequest.zeroState(c).withMeasurement(MeasurementInstruction.countsAll(32))
    with pytest.raises(A.UnsupportedOperationException):
        fused.simulate(req)


# ---- random circuits vs the oracle --------------------------------------------
@pytest.mark.parametrize("n", [1, 2, 3, 4, 6, 9, 12, 15, 18])
def test_random_circuits_match_oracle(n, fused, unfused):
    for seed in range(3):
        c = RCirc.random_circuit(n, 60, seed=31 * n + seed)
        init = RCirc.random_state(n, seed)
        want = _oracle_state(c, init)
        req = SimulationRequest.withInitialState(c, Q.StateVector.fromArray(n, init))
        for engine in (fused, unfused):
            got = engine.simulate(req).finalState.data()
            np.testing.assert_allclose(got, want, rtol=0, atol=EPS)


@pytest.mark.parametrize("cfg", [dict(tile_qubits=8), dict(tile_qubits=10, sweep_budget=-1),
                                 dict(tile_qubits=12, sweep_budget=16)])
def test_tile_configurations_agree(cfg):
    n = 16
    c = RCirc.random_circuit(n, 200, seed=5)
    want = _oracle_state(c)
    e = StatevectorB200Engine(B200Config(**cfg))
    got = e.simulate(SimulationRequest.zeroState(c)).finalState.data()
    e.close()
    np.testing.assert_allclose(got, want, rtol=0, atol=EPS)


def test_brickwall_20q_matches_oracle_and_counts(fused):
    """20-qubit brick-wall U3 + CNOT, 20 layers, countsAll(1024) seed 42."""
    c = W.brickwall_circuit(20, 20, seed=2020)
    want = _oracle_state(c)
    req = (SimulationRequest.zeroState(c)
           .withMeasurement(MeasurementInstruction.countsAll(1024).withSeed(42), True))
    res = fused.simulate(req)
    got = res.finalState.data()
    np.testing.assert_allclose(got, want, rtol=0, atol=EPS)
    want_out = O.sample(want, 20, list(range(20)), 1024, 42)
    want_counts = {int(k): int(v) for k, v in zip(*np.unique(want_out, return_counts=True))}
    if res.measurement.counts != want_counts:
        # allowed only for draws within the CDF error band of a boundary
        u = O.uniforms(42, 1024)
        cdf = O.cumulative(O.probabilities(want, 20, list(range(20))))
        gpu_out = fused.context().sample(list(range(20)), 1024, 42)
        for k in np.nonzero(gpu_out != want_out)[0]:
            j = int(want_out[k])
            lo = cdf[j - 1] if j > 0 else 0.0
            assert min(abs(u[k] - lo), abs(u[k] - cdf[j])) < 1e-12


# ---- sampling -----------------------------------------------------------------
@pytest.mark.parametrize("n,m_qubits", [(10, None), (12, (0, 5, 11)), (14, (13,)), (16, None)])
def test_sampling_bit_exact_on_shared_uniforms(n, m_qubits, fused):
    init = RCirc.random_state(n, 11)
    qubits = list(range(n)) if m_qubits is None else list(m_qubits)
    ctx = fused.context()
    ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), init)
    shots = 4096
    u = O.uniforms(1234, shots)
    gpu = ctx.sample(qubits, shots, None, u)
    cpu = O.sample(init, n, qubits, shots, 0, u)
    cdf = O.cumulative(O.probabilities(init, n, qubits))
    mism = np.nonzero(gpu != cpu)[0]
    for k in mism:
        j = int(cpu[k])
        edges = [cdf[j - 1] if j > 0 else 0.0, cdf[j]]
        assert min(abs(u[k] - e) for e in edges) < 1e-12, (k, gpu[k], cpu[k])
    assert len(mism) <= 2
    # the seeded path draws SplittableRandom(seed).nextDouble() per shot
    np.testing.assert_array_equal(ctx.sample(qubits, shots, 1234), gpu)


@pytest.mark.parametrize("scale", [1.0, 1.5, 0.25 + 1e-9])
def test_sampling_reproduces_the_reference_running_sum(scale, fused):
    # the running sum of 2^16 probabilities, with the reference's rescaling when the
    # total is off by more than 1e-12 (scale != 1): outcomes identical on shared
    # uniforms, including draws placed exactly on CDF entries and half-way ties
    n = 16
    init = RCirc.random_state(n, 21) * math.sqrt(scale)
    ctx = fused.context()
    ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), init)
    cdf = O.cumulative(O.probabilities(init, n, list(range(n))))
    rng = np.random.default_rng(3)
    u = np.concatenate([rng.random(3000), cdf[rng.integers(0, cdf.size - 1, 500)],
                        np.nextafter(cdf[rng.integers(0, cdf.size - 1, 500)], 0)])
    got = ctx.sample(list(range(n)), u.size, None, u)
    want = O.sample(init, n, list(range(n)), u.size, 0, u)
    np.testing.assert_array_equal(got, want)


def test_sampling_dyadic_probabilities_with_ties(fused):
    # probabilities that are sums of few powers of two make the running sum hit
    # half-way cases of round-to-nearest-even; a state of 2^18 such entries
    n = 18
    rng = np.random.default_rng(8)
    p = rng.choice([0.0, 2.0 ** -18, 2.0 ** -20, 3 * 2.0 ** -21, 2.0 ** -40], size=1 << n)
    p[-1] += 1.0 - p.sum()
    init = np.zeros(2 << n)
    init[0::2] = np.sqrt(np.maximum(p, 0.0))
    ctx = fused.context()
    ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), init)
    cdf = O.cumulative(O.probabilities(init, n, list(range(n))))
    u = np.concatenate([rng.random(4000), cdf[rng.integers(0, cdf.size - 1, 1000)]])
    got = ctx.sample(list(range(n)), u.size, None, u)
    want = O.sample(init, n, list(range(n)), u.size, 0, u)
    np.testing.assert_array_equal(got, want)


def _sparse_probabilities(kind, n, rng):
    p = np.zeros(1 << n)
    if kind == "ghz":
        p[0] = p[-1] = 0.5
    elif kind == "last":
        p[-1] = 1.0
    elif kind == "middle":
        p[rng.integers(17 * 2048, 18 * 2048, 5)] = rng.random(5)
    elif kind == "tiny_head":
        p[:300] = 1e-300
        p[300:310] = rng.random(10)
        p[5000:5003] = 2.0 ** -1070  # subnormal steps on a normal sum
    elif kind == "zero_chunks":
        keep = rng.random((1 << n) // 2048) < 0.1
        p = rng.random(1 << n) * np.repeat(keep, 2048)
    return p / p.sum()


@pytest.mark.parametrize("kind", ["ghz", "last", "middle", "tiny_head", "zero_chunks"])
def test_sampling_sparse_states(kind, fused):
    # chunks of zeros before, between and after the mass; a running sum that starts
    # at tiny values; all the mass in the last chunk
    n = 16
    rng = np.random.default_rng(31)
    p = _sparse_probabilities(kind, n, rng)
    init = np.zeros(2 << n)
    init[0::2] = np.sqrt(p)
    ctx = fused.context()
    ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), init)
    cdf = O.cumulative(O.probabilities(init, n, list(range(n))))
    nz = np.flatnonzero(np.diff(np.concatenate([[0.0], cdf])))
    u = np.concatenate([rng.random(3000), cdf[nz], np.nextafter(cdf[nz], 0), [0.0]])
    got = ctx.sample(list(range(n)), u.size, None, u)
    want = O.sample(init, n, list(range(n)), u.size, 0, u)
    np.testing.assert_array_equal(got, want)


def test_tie_rule_and_last_entry(fused):
    # state with exact probabilities 1/4, 0, 1/4, 1/2 on 2 qubits
    init = np.array([0.5, 0, 0, 0, 0.5, 0, math.sqrt(0.5), 0])
    ctx = fused.context()
    ctx.run_ops(2, *serialize_circuit(Q.QuantumCircuit(2)), init)
    u = np.array([0.0, 0.25, 0.2500000001, 0.5, 0.75, 0.999999, 1.0, 5.0])
    got = ctx.sample([0, 1], u.size, None, u)
    cdf = O.cumulative(O.probabilities(init, 2, [0, 1]))
    want = [O.sample_outcome(cdf, float(x)) for x in u]
    assert got.tolist() == want


def test_probabilities_match_reference_order(fused):
    n = 12
    init = RCirc.random_state(n, 2)
    ctx = fused.context()
    ctx.run_ops(n, *serialize_circuit(Q.QuantumCircuit(n)), init)
    for qubits in ([3], [0, 7, 11], list(range(n))):
        got = ctx.probabilities(qubits)
        p = O.probabilities(init, n, qubits)
        s = float(np.sum(p))
        want = p / s if abs(s - 1.0) > 1e-12 else p
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-15)


def test_zero_state_sampling_raises(fused):
    ctx = fused.context()
    ctx.run_ops(3, *serialize_circuit(Q.QuantumCircuit(3)), np.zeros(16))
    with pytest.raises(A.IllegalStateException):
        ctx.sample([0, 1, 2], 8, 1)


def test_bell_histogram_balanced(fused):
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
    req = SimulationRequest.zeroState(c).withMeasurement(
        MeasurementInstruction.countsAll(10_000).withSeed(0xCAFEBABE))
    h = fused.simulate(req).measurement
    assert h.measuredQubits == (0, 1)
    assert h.counts.get(0, 0) + h.counts.get(3, 0) == 10_000
    assert abs(h.counts.get(0, 0) - 5000) <= 400


def test_measure_ops_define_default_targets(fused):
    c = Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.PauliX(), 2).measure(0, 2)
    req = SimulationRequest.zeroState(c).withMeasurement(
        MeasurementInstruction.countsAll(1000).withSeed(42))
    h = fused.simulate(req).measurement
    assert h.measuredQubits == (0, 2)
    assert sum(h.counts.values()) == 1000


# ---- noise --------------------------------------------------------------------
def _noise_cases():
    c1 = Q.QuantumCircuit(1).append(Q.PauliX(), 0)
    yield "depolarizing", c1, NoiseModel.builder().afterAllGates(ErrorChannel.depolarizing(1.0, 0)).build(), 77
    yield "amp_damping", c1, NoiseModel.builder().afterAllGates(ErrorChannel.amplitudeDamping(0.4, 0)).build(), 123
    yield "thermal", c1, NoiseModel.builder().afterAllGates(ErrorChannel.thermalRelaxation(1e-6, 2e-6, 1e-3, 0)).build(), 9
    c5 = (Q.QuantumCircuit(5).append(Q.Hadamard(), 0).append(Q.Hadamard(), 3)
          .append(Q.CnotGate.of(), 3, 1).appendSwap(0, 4).appendControlledPhase(math.pi / 5.0, 4, 2)
          .appendMultiControl(Q.PauliX(), 2, 0, 1, 3))
    yield "mixed_phase_amp", c5, (NoiseModel.builder()
                                  .afterAllGates(ErrorChannel.phaseFlip(0.35, 0))
                                  .afterAllGates(ErrorChannel.amplitudeDamping(0.2, 3)).build()), 99
    c12 = RCirc.random_circuit(12, 40, seed=3)
    model = (NoiseModel.builder().afterAllGates(ErrorChannel.depolarizing(0.05, 4))
             .onQubits(ErrorChannel.phaseDamping(0.1, 0), 2, 7)
             .afterGate(Q.CnotOperation, ErrorChannel.amplitudeDamping(0.1, 9)).build())
    yield "random_12q", c12, model, 2024


@pytest.mark.parametrize("case", list(_noise_cases()), ids=lambda c: c[0])
def test_noisy_runs_match_oracle(case, fused):
    _, c, model, seed = case
    req = SimulationRequest.zeroState(c).withNoiseModel(model).withNoiseSeed(seed)
    want, _, _ = O.simulate_request(req)
    got = fused.simulate(req).finalState.data()
    np.testing.assert_allclose(got, want, rtol=0, atol=EPS)


def test_noise_goldens(fused):
    inv = 1.0 / math.sqrt(2.0)
    model = NoiseModel.builder().afterAllGates(ErrorChannel.phaseFlip(1.0, 0)).build()
    st = fused.simulate(SimulationRequest.zeroState(Q.QuantumCircuit(1).append(Q.Hadamard(), 0))
                        .withNoiseModel(model)).finalState.data()
    np.testing.assert_allclose(st, [inv, 0, -inv, 0], atol=EPS)
    model = NoiseModel.builder().afterAllGates(ErrorChannel.amplitudeDamping(1.0, 0)).build()
    req = (SimulationRequest.zeroState(Q.QuantumCircuit(1).append(Q.PauliX(), 0)).withNoiseModel(model)
           .withMeasurement(MeasurementInstruction.countsAll(16).withSeed(5), False))
    assert fused.simulate(req).measurement.counts == {0: 16}


def test_invalid_noise_qubit_throws(fused):
    model = NoiseModel.builder().afterAllGates(ErrorChannel.phaseFlip(0.1, 2)).build()
    req = SimulationRequest.zeroState(Q.QuantumCircuit(1).append(Q.Hadamard(), 0)).withNoiseModel(model)
    with pytest.raises(ValueError):
        fused.simulate(req)


# ---- complex64 ------------------------------------------------------------------
@pytest.mark.parametrize("n", [3, 10, 16])
def test_complex64_error_vs_complex128(n, c64):
    c = RCirc.random_circuit(n, 80, seed=n)
    want = _oracle_state(c)
    got = c64.simulate(SimulationRequest.zeroState(c)).finalState.data()
    assert np.max(np.abs(got - want)) < 2e-5


def _near_pi_chain(n, u00, gates, seed):
    # H on every qubit, then a long chain of u3 gates with |u00| = u00 (and a few
    # CNOTs): the rotation-form scalars of the chain multiply to far below the
    # floating-point range unless the sweeps apply them in time
    c = Q.QuantumCircuit(n)
    for q in range(n):
        c = c.append(Q.Hadamard(), q)
    rng = np.random.default_rng(seed)
    theta = 2 * math.acos(u00)
    for _ in range(gates):
        q = int(rng.integers(0, n))
        c = c.append(Q.u3(theta, float(rng.uniform(0, 6.3)), float(rng.uniform(0, 6.3))), q)
        if rng.random() < 0.1:
            c = c.append(Q.CnotGate.of(), q, (q + 1) % n)
    return c


@pytest.mark.parametrize("n", [12, 20])
def test_rotation_form_scalar_stays_in_range(n, fused, c64):
    c = _near_pi_chain(n, 0.06, 600, n)
    want = _oracle_state(c)
    got = fused.simulate(SimulationRequest.zeroState(c)).finalState.data()
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(got, want, rtol=0, atol=EPS)
    c = _near_pi_chain(n, 0.26, 600, n + 1)
    want = _oracle_state(c)
    got = c64.simulate(SimulationRequest.zeroState(c)).finalState.data()
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - want)) < 2e-5


# ---- expectation values / adjoint ---------------------------------------------
def test_pauli_expectation_matches_oracle(fused):
    n = 10
    c = RCirc.random_circuit(n, 50, seed=8)
    st = _oracle_state(c)
    fused.simulate(SimulationRequest.zeroState(c))
    x, z, coef = W.random_pauli_sum(n, 16, seed=6464)
    got = fused.context().expect_pauli(x, z, coef)
    want = O.expect_pauli(st, n, x, z, coef)
    assert got == pytest.approx(want, abs=1e-12)


def _param_shift(n, ops, n_ops, params, x, z, c):
    grad = np.zeros(params.size)
    for k in range(params.size):
        vals = []
        for s in (+math.pi / 2, -math.pi / 2):
            p = params.copy()
            p[k] += s
            st = O.initial_state(n)
            rc, _ = O.run(n, ops, n_ops, st, params=p)
            assert rc == 0
            vals.append(O.expect_pauli(st, n, x, z, c))
        grad[k] = 0.5 * (vals[0] - vals[1])
    return grad


@pytest.mark.parametrize("n,layers", [(6, 3), (12, 2)])
def test_adjoint_gradient_matches_parameter_shift(n, layers):
    from statecraft_b200.adjoint import AdjointEngine

    ops, n_ops, n_params = W.hea_ops(n, layers)
    params = W.hea_params(n_params, seed=2626)
    x, z, c = W.random_pauli_sum(n, 12, seed=6464)
    eng = AdjointEngine()
    e, g = eng.value_and_grad(n, ops, n_ops, params, x, z, c)
    st = O.initial_state(n)
    O.run(n, ops, n_ops, st, params=params)
    assert e == pytest.approx(O.expect_pauli(st, n, x, z, c), abs=1e-12)
    ps = _param_shift(n, ops, n_ops, params, x, z, c)
    np.testing.assert_allclose(g, ps, rtol=0, atol=1e-8)
    eng.close()


def test_adjoint_gradient_matches_central_differences():
    # the FP64 check of the adjoint method against central finite differences (h = 1e-6)
    # on the plain forward engine; FD round-off sets the tolerance
    from statecraft_b200.adjoint import AdjointEngine

    n, layers, h = 14, 3, 1e-6
    ops, n_ops, n_params = W.hea_ops(n, layers)
    params = W.hea_params(n_params, seed=2626)
    x, z, c = W.random_pauli_sum(n, 24, seed=6464)
    eng = AdjointEngine()
    _, g = eng.value_and_grad(n, ops, n_ops, params, x, z, c)
    fd = np.zeros(n_params)
    for k in range(n_params):
        vals = []
        for s in (h, -h):
            p = params.copy()
            p[k] += s
            vals.append(eng.expectation(n, ops, n_ops, p, x, z, c))
        fd[k] = (vals[0] - vals[1]) / (2 * h)
    noise = 4 * np.finfo(float).eps * float(np.sum(np.abs(c))) * n_ops / h
    np.testing.assert_allclose(g, fd, rtol=0, atol=max(1e-8, noise))
    eng.close()


def test_adjoint_complex64_error_reported():
    from statecraft_b200.adjoint import AdjointEngine

    n, layers = 12, 3
    ops, n_ops, n_params = W.hea_ops(n, layers)
    params = W.hea_params(n_params, seed=2626)
    x, z, c = W.random_pauli_sum(n, 16, seed=6464)
    e128 = AdjointEngine()
    e64 = AdjointEngine(B200Config(dtype=A.SC_C64))
    v1, g1 = e128.value_and_grad(n, ops, n_ops, params, x, z, c)
    v2, g2 = e64.value_and_grad(n, ops, n_ops, params, x, z, c)
    err = float(np.max(np.abs(g1 - g2)))
    print("complex64 adjoint: |dE| = %.3e, max |d grad| = %.3e" % (abs(v1 - v2), err))
    assert abs(v1 - v2) < 1e-4 and err < 1e-4
    e128.close()
    e64.close()


# ---- full-size properties ---------------------------------------------------------
def test_28q_brickwall_fused_matches_unfused():
    c = W.brickwall_circuit(28, 4, seed=3030, mcz=True, rzz=True)
    a = StatevectorB200Engine(B200Config(fusion=True))
    a.simulate(SimulationRequest.zeroState(c))
    sa = a.final_state_array()
    a.close()
    b = StatevectorB200Engine(B200Config(fusion=False))
    b.simulate(SimulationRequest.zeroState(c))
    sb = b.final_state_array()
    b.close()
    assert np.max(np.abs(sa - sb)) < 1e-12
    assert float(np.dot(sa, sa)) == pytest.approx(1.0, abs=1e-10)


def test_memory_limit_reports_enomem():
    e = StatevectorB200Engine(B200Config(device_mem_limit=1 << 20))
    with pytest.raises(A.EngineError) as info:
        e.simulate(SimulationRequest.zeroState(Q.QuantumCircuit(20)))
    assert info.value.status == A.SC_ENOMEM
    e.close()


@pytest.mark.parametrize("dtype,tol", [(A.SC_C128, 1e-12), (A.SC_C64, 2e-6)])
def test_32_qubit_maximum_size(dtype, tol):
    # the largest register the engine takes (2^32 amplitudes: 64 GiB c128, 32 GiB c64),
    # where every tile and amplitude index uses the full 32 bits: GHZ-32, X on qubit
    # 0, RY(1) on qubit 31; marginals and seeded samples against the closed form
    n = 32
    c = Q.QuantumCircuit(n).append(Q.Hadamard(), 0)
    for q in range(n - 1):
        c = c.append(Q.CnotGate.of(), q, q + 1)
    c = c.append(Q.PauliX(), 0).append(Q.ry(1.0), n - 1)
    ops, n_ops = serialize_circuit(c)
    ctx = NativeContext(B200Config(dtype=dtype))
    try:
        ctx.run_ops(n, ops, n_ops)
        cs, sn = math.cos(0.5) ** 2 / 2, math.sin(0.5) ** 2 / 2
        np.testing.assert_allclose(ctx.probabilities([0, n - 1]), [sn, cs, cs, sn], rtol=0, atol=tol)
        want = np.zeros(8)
        want[0], want[7] = 0.5, 0.5  # qubits 5, 17, 26 follow the GHZ branches
        np.testing.assert_allclose(ctx.probabilities([5, 17, 26]), want, rtol=0, atol=tol)
        shots = ctx.sample([0, n - 1], 8192, 2024)
        counts = np.bincount(shots, minlength=4)
        assert np.all(np.abs(counts - 8192 * np.array([sn, cs, cs, sn])) < 6 * np.sqrt(8192 * 0.25))
    finally:
        ctx.close()
