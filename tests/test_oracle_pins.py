"""Pins the CPU oracle before anything is checked against it.

- SplitMix64 (java.util.SplittableRandom) against its published output sequence.
- The oracle engine against the reference's naive evaluator on every circuit of
  StatevectorEngineTest (1e-12, the reference tests' EPS).
- The deterministic noise goldens and statistics of StatevectorNoiseTest.
- Measurement semantics: CDF rule, tie rule, u >= 1, Bell balance.
- LASSQ norm (ComplexArrays.norm2Sq) edge cases.
"""
import math

import numpy as np
import pytest

import refcircuits as RC
from java_random import JavaRandom
from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import quantum as Q
from statecraft_b200.engine import MeasurementInstruction, SimulationRequest
from statecraft_b200.noise import ErrorChannel, NoiseModel

EPS = 1e-12


def test_splitmix64_published_sequence():
    # splitmix64 reference outputs for seed 1234567 (Vigna's splitmix64.c)
    r = O.SplittableRandom(1234567)
    assert [r.nextLong() for _ in range(5)] == [
        6457827717110365317, 3203168211198807973, 9817491932198370423,
        4593380528125082431, 16408922859458223821]


def test_next_double_is_top_53_bits():
    a, b = O.SplittableRandom(99), O.SplittableRandom(99)
    for _ in range(100):
        assert a.nextDouble() == (b.nextLong() >> 11) * 2.0 ** -53


def test_next_double_bound_stays_below_bound():
    r = O.SplittableRandom(7)
    for bound in (1e-300, 0.5, 1.0, 3.0, 1e300):
        for _ in range(50):
            v = r.nextDouble(bound)
            assert 0.0 <= v < bound


def test_java_util_random_known_values():
    assert JavaRandom(42).nextInt() == -1170105035
    assert JavaRandom(0).nextDouble() == 0.730967787376657


@pytest.mark.parametrize("name", [c[0] for c in RC.cases()])
def test_oracle_matches_naive_reference(name):
    case = {c[0]: c for c in RC.cases()}[name]
    _, request, expected = case
    st, _, _ = O.simulate_request(request)
    np.testing.assert_allclose(st, RC.to_interleaved(expected), rtol=0, atol=EPS)


def test_oracle_22_qubit_basis_kat():
    request, idx = RC.large_basis_case()
    st, _, _ = O.simulate_request(request)
    assert st[2 * idx] == pytest.approx(1.0, abs=EPS)
    assert st[2 * idx + 1] == pytest.approx(0.0, abs=EPS)
    assert O.norm2sq(st) == pytest.approx(1.0, abs=1e-10)


def test_unitary_after_measure_rejected():
    # unitaryAfterMeasurementThrows (StatevectorEngineTest.java:333-343)
    c = Q.QuantumCircuit(1).append(Q.Hadamard(), 0).measure(0).append(Q.PauliX(), 0)
    req = SimulationRequest.zeroState(c).withMeasurement(MeasurementInstruction.countsAll(32))
    with pytest.raises(A.UnsupportedOperationException):
        O.simulate_request(req)


# ---- noise goldens (StatevectorNoiseTest.java) --------------------------------
INV_SQRT2 = 1.0 / math.sqrt(2.0)


def _noisy(c, model, seed=None, basis=None, init=None):
    req = SimulationRequest.zeroState(c) if init is None else SimulationRequest.withInitialState(c, init)
    if basis is not None:
        req = req.withBasisState(*basis)
    req = req.withNoiseModel(model)
    if seed is not None:
        req = req.withNoiseSeed(seed)
    return req


def test_phase_flip_on_plus_applies_z():  # :40-51
    model = NoiseModel.builder().afterAllGates(ErrorChannel.phaseFlip(1.0, 0)).build()
    st, _, _ = O.simulate_request(_noisy(Q.QuantumCircuit(1).append(Q.Hadamard(), 0), model))
    np.testing.assert_allclose(st, [INV_SQRT2, 0, -INV_SQRT2, 0], atol=EPS)


def test_depolarizing_seed_deterministic_and_normalized():  # :53-67
    model = NoiseModel.builder().afterAllGates(ErrorChannel.depolarizing(1.0, 0)).build()
    c = Q.QuantumCircuit(1).append(Q.PauliX(), 0)
    a, _, _ = O.simulate_request(_noisy(c, model, 77))
    b, _, _ = O.simulate_request(_noisy(c, model, 77))
    np.testing.assert_array_equal(a, b)
    assert O.norm2sq(a) == pytest.approx(1.0, abs=EPS)


def test_amplitude_damping_distribution():  # :85-106
    gamma = 0.25
    model = NoiseModel.builder().afterAllGates(ErrorChannel.amplitudeDamping(gamma, 0)).build()
    c = Q.QuantumCircuit(1).append(Q.PauliX(), 0)
    zeros = 0
    for trial in range(1000):
        st, _, _ = O.simulate_request(_noisy(c, model, 0xBAD0 + trial))
        if st[0] ** 2 + st[1] ** 2 > 0.5:
            zeros += 1
    assert zeros / 1000 == pytest.approx(gamma, abs=0.05)


def test_idle_decoherence_uses_mapped_qubit():  # :117-128
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0)
    init = Q.StateVector.fromArray(2, [0, 0, 0, 0, 0, 0, 1, 0])
    model = NoiseModel.builder().onQubits(ErrorChannel.amplitudeDamping(1.0, 0), 0, 1).build()
    st, _, _ = O.simulate_request(_noisy(c, model, init=init))
    np.testing.assert_allclose(st, [INV_SQRT2, 0, -INV_SQRT2, 0, 0, 0, 0, 0], atol=EPS)


@pytest.mark.parametrize("channel", [ErrorChannel.amplitudeDamping(0.9, 1),
                                     ErrorChannel.phaseDamping(0.9, 1)])
def test_ground_state_skips_zero_branch(channel):  # :141-165
    model = NoiseModel.builder().afterAllGates(channel).build()
    st, _, _ = O.simulate_request(_noisy(Q.QuantumCircuit(2).append(Q.Hadamard(), 0), model, 3))
    np.testing.assert_allclose(st, [INV_SQRT2, 0, INV_SQRT2, 0, 0, 0, 0, 0], atol=EPS)


def test_scheduled_noise_paths_golden():  # :167-181
    model = (NoiseModel.builder()
             .afterGate(Q.SingleGateOperation, ErrorChannel.phaseFlip(1.0, 0))
             .onQubits(ErrorChannel.amplitudeDamping(1.0, 0), 1)
             .afterAllGates(ErrorChannel.phaseFlip(1.0, 0)).build())
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0)
    st, _, _ = O.simulate_request(_noisy(c, model, basis=(0, 1)))
    np.testing.assert_allclose(st, [INV_SQRT2, 0, -INV_SQRT2, 0, 0, 0, 0, 0], atol=EPS)


def test_noisy_measurement_histogram_golden():  # :183-194
    model = NoiseModel.builder().afterAllGates(ErrorChannel.amplitudeDamping(1.0, 0)).build()
    c = Q.QuantumCircuit(1).append(Q.PauliX(), 0)
    req = (SimulationRequest.zeroState(c).withNoiseModel(model)
           .withMeasurement(MeasurementInstruction.countsAll(16).withSeed(5), False))
    _, meas, _ = O.simulate_request(req)
    assert np.bincount(meas["outcomes"], minlength=2).tolist() == [16, 0]


def test_thermal_relaxation_to_ground():  # :196-207
    model = NoiseModel.builder().afterAllGates(
        ErrorChannel.thermalRelaxation(1e-6, 2e-6, 1e-3, 0)).build()
    st, _, _ = O.simulate_request(_noisy(Q.QuantumCircuit(1).append(Q.PauliX(), 0), model, 9))
    np.testing.assert_allclose(st, [1, 0, 0, 0], atol=EPS)
    assert O.norm2sq(st) == pytest.approx(1.0, abs=EPS)


# ---- measurement ----------------------------------------------------------------
def test_bell_histogram_balanced():  # :257-279
    c = Q.QuantumCircuit(2).append(Q.Hadamard(), 0).append(Q.CnotGate.of(), 0, 1)
    req = SimulationRequest.zeroState(c).withMeasurement(
        MeasurementInstruction.countsAll(10_000).withSeed(0xCAFEBABE))
    _, meas, _ = O.simulate_request(req)
    counts = np.bincount(meas["outcomes"], minlength=4)
    assert counts[0] + counts[3] == 10_000
    assert abs(counts[0] - 5000) <= 400 and abs(counts[3] - 5000) <= 400


def test_cdf_rules():
    cdf = O.cumulative(np.array([0.25, 0.0, 0.25, 0.5]))
    assert cdf.tolist() == [0.25, 0.25, 0.5, 1.0]
    # ties walk left; exact boundary selects the first index reaching it
    assert O.sample_outcome(cdf, 0.25) == 0
    assert O.sample_outcome(cdf, 0.2500000001) == 2
    assert O.sample_outcome(cdf, 0.0) == 0
    assert O.sample_outcome(cdf, 0.75) == 3
    assert O.sample_outcome(cdf, 1.0) == 3
    assert O.sample_outcome(cdf, 7.0) == 3


def test_normalize_rescales_only_outside_tolerance():
    cdf = O.cumulative(np.array([1.0, 1.0]))
    assert cdf.tolist() == [0.5, 1.0]
    with pytest.raises(RuntimeError):
        O.cumulative(np.zeros(4))


def test_partial_measurement_marginals():
    # partialMeasurementTargetsSpecifiedQubits (:281-301)
    c = (Q.QuantumCircuit(3).append(Q.Hadamard(), 0).append(Q.Hadamard(), 1)
         .append(Q.CnotGate.of(), 0, 2))
    st, _, _ = O.simulate_request(SimulationRequest.zeroState(c))
    p = O.probabilities(st, 3, [2])
    np.testing.assert_allclose(p, [0.5, 0.5], atol=EPS)


# ---- LASSQ norm ------------------------------------------------------------------
def test_lassq_norm_edges():
    assert O.norm2sq(np.zeros(8)) == 0.0
    assert math.isnan(O.norm2sq(np.array([1.0, float("nan")])))
    assert O.norm2sq(np.array([float("inf"), 0.0])) == float("inf")
    # LASSQ keeps the running sum scaled; only the final scale^2 * ssq can overflow
    assert O.norm2sq(np.array([1e150, 1e150, 0.0, 0.0])) == pytest.approx(2e300, rel=1e-15)
    assert O.norm2sq(np.array([1e200, 1e200, 1e200, 0.0])) == float("inf")
    assert O.norm2sq(np.array([3e-160, 0.0, 4e-160, 0.0])) == pytest.approx(25e-320, rel=1e-3)
    x = np.random.default_rng(1).standard_normal(64)
    assert O.norm2sq(x) == pytest.approx(float(np.sum(x * x)), rel=1e-14)


def test_expectation_matches_dense_algebra():
    rng = np.random.default_rng(3)
    n = 4
    amps = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    amps /= np.linalg.norm(amps)
    st = np.empty(32)
    st[0::2], st[1::2] = amps.real, amps.imag
    X = np.array([[0, 1], [1, 0]], dtype=complex)
    Y = np.array([[0, -1j], [1j, 0]])
    Z = np.diag([1.0 + 0j, -1.0])
    I2 = np.eye(2, dtype=complex)
    for _ in range(20):
        letters = rng.integers(0, 4, n)
        xm = zm = 0
        mat = np.array([[1.0 + 0j]])
        for q in range(n):  # little-endian: qubit q is bit q, kron puts q=n-1 first
            L = int(letters[q])
            if L in (1, 2):
                xm |= 1 << q
            if L in (2, 3):
                zm |= 1 << q
            mat = np.kron((I2, X, Y, Z)[L], mat)
        want = float(np.real(np.vdot(amps, mat @ amps)))
        got = O.expect_pauli(st, n, [xm], [zm], [1.0])
        assert got == pytest.approx(want, abs=1e-13)


def test_qaoa_ring_energy_popcount_form():
    # The batched QAOA kernels evaluate sum_j Z_j Z_{j+1 mod n} on basis state x as
    # n - 2 popcount(x XOR rotr_n(x)) and fold a layer's ring phases into
    # exp(-i gamma (n - 2k)); both identities checked on the oracle.
    from statecraft_b200 import workloads as W
    from statecraft_b200.engine import serialize_circuit

    n = 7
    rng = np.random.default_rng(5)
    st = rng.normal(size=2 << n)
    st /= np.sqrt(np.sum(st ** 2))
    z = [(1 << j) | (1 << ((j + 1) % n)) for j in range(n)]
    direct = O.expect_pauli(st, n, [0] * n, z, [1.0] * n)
    probs = st[0::2] ** 2 + st[1::2] ** 2
    x = np.arange(1 << n)
    rot = (x >> 1) | ((x & 1) << (n - 1))
    k = np.array([bin(v).count("1") for v in (x ^ rot)])
    assert abs(direct - np.sum(probs * (n - 2 * k))) < 1e-12
    # one layer of ring phases from |+>^n equals the tabulated phase per basis state
    g = 0.37
    c = W.qaoa_circuit(n, [g], [0.0])
    ops, n_ops = serialize_circuit(c)
    s2 = O.initial_state(n)
    assert O.run(n, ops, n_ops, s2)[0] == 0
    amp = s2[0::2] + 1j * s2[1::2]
    want = np.exp(-1j * g * (n - 2 * k)) / np.sqrt(2.0 ** n)
    np.testing.assert_allclose(amp, want, rtol=0, atol=1e-14)
