"""Batched QAOA ring ansatz on the GPU against the oracle, gate by gate.

Bar: complex128 energies within 1e-10 of the oracle's FP64 gate-by-gate result
(each instance is O(n) in magnitude; the kernel folds a layer's n ZZ phases into
one table entry, a different rounding path); norms within 1e-12 of 1; the
complex64 path's energy error against complex128 is reported per instance and
must stay below 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as O
from statecraft_b200 import _abi as A
from statecraft_b200 import workloads as W
from statecraft_b200.batch import QaoaRingBatch
from statecraft_b200.engine import B200Config, NativeContext

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = NativeContext(B200Config())
    yield c
    c.close()


def _instances(count, p, seed, n_min, n_max):
    b = W.qaoa_instances(count, p, seed, n_min=n_min, n_max=n_max)
    return b.n_qubits, b.gammas, b.betas


@pytest.mark.parametrize("p", [1, 2, 4])
def test_batch_matches_oracle(ctx, p):
    nq, g, b = _instances(48, p, 4000 + p, 2, 17)   # whole (<= 12) and split (13..17) instances
    batch = QaoaRingBatch(nq, g, b, context=ctx)
    batch.run()
    e, norms = batch.energies(with_norms=True)
    want = np.array([O.qaoa_ring_energy(int(n), g[i], b[i]) for i, n in enumerate(nq)])
    np.testing.assert_allclose(e, want, rtol=0, atol=1e-10)
    np.testing.assert_allclose(norms, 1.0, rtol=0, atol=1e-12)
    batch.close()


def test_largest_instances_match_oracle(ctx):
    nq = np.array([23, 20, 22, 12, 13], dtype=np.int32)
    rng = W.SplitMix64(99)
    g = np.array([[rng.nextDouble(np.pi) for _ in range(4)] for _ in nq])
    b = np.array([[rng.nextDouble(np.pi) for _ in range(4)] for _ in nq])
    batch = QaoaRingBatch(nq, g, b, context=ctx)
    e = batch.evaluate()
    want = np.array([O.qaoa_ring_energy(int(n), g[i], b[i]) for i, n in enumerate(nq)])
    np.testing.assert_allclose(e, want, rtol=0, atol=1e-10)
    batch.close()


def test_complex64_error_reported_and_small(ctx):
    nq, g, b = _instances(64, 4, 77, 10, 18)
    e128 = QaoaRingBatch(nq, g, b, context=ctx).evaluate()
    b64 = QaoaRingBatch(nq, g, b, dtype=A.SC_C64, context=ctx)
    b64.run()
    e64, n64 = b64.energies(with_norms=True)
    err = np.abs(e64 - e128)
    print("complex64 energy error vs complex128: max %.3e mean %.3e" % (err.max(), err.mean()))
    assert err.max() < 1e-4
    np.testing.assert_allclose(n64, 1.0, rtol=0, atol=1e-5)


def test_shapes_agree_and_angles_update(ctx):
    nq, g, b = _instances(32, 3, 5, 8, 16)
    tuned = QaoaRingBatch(nq, g, b, tune=True, context=ctx)
    fixed = QaoaRingBatch(nq, g, b, tune=False, context=ctx)
    np.testing.assert_allclose(tuned.evaluate(), fixed.evaluate(), rtol=0, atol=1e-12)
    info = tuned.info()
    assert info["register_qubits"] in (3, 4) and info["ctas_per_sm"] >= 1
    # new angles through the captured graph equal a fresh batch built with them
    g2, b2 = g[::-1].copy(), b[::-1].copy()
    tuned.set_angles(g2, b2)
    fresh = QaoaRingBatch(nq, g2, b2, tune=False, context=ctx)
    np.testing.assert_allclose(tuned.evaluate(), fresh.evaluate(), rtol=0, atol=1e-12)
    for x in (tuned, fixed, fresh):
        x.close()


def test_invalid_batches_rejected(ctx):
    with pytest.raises(A.IllegalArgumentException):
        QaoaRingBatch([24], [[0.1]], [[0.2]], context=ctx)
    with pytest.raises(A.IllegalArgumentException):
        QaoaRingBatch([1], [[0.1]], [[0.2]], context=ctx)
    with pytest.raises(A.IllegalArgumentException):
        QaoaRingBatch([4], np.zeros((1, 17)), np.zeros((1, 17)), context=ctx)
