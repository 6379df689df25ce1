/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference `statevector` engine, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * Nothing in the product (statecraft_b200/) links, loads or calls this file.
 *
 * Sources restated (paths within the StateCraft project):
 *   engines/src/main/java/com/omaarr90/statecraft/engines/statevector/StatevectorOps.java
 *       scalar paths of applySingleGate (:62-82), applyCnot (:128-145),
 *       applyTwoQubitUnitary (:335-383), applyTwoQubitDiagonal (:480-517),
 *       applySwap (:576-593), applyMultiControlledSingleGate (:678-701)
 *   engines/.../statevector/StatevectorEngine.java
 *       simulate op loop (:63-151), computeMeasurementProbabilities (:274-296),
 *       normalize (:298-312), cumulative (:314-323), sampleOutcome (:325-338),
 *       sampleKrausOperator / computeBranchWeight / applyKrausMatrix /
 *       blockNormSquared / sampleWeightedIndex / renormalizeState (:463-600)
 *   core/.../core/math/ComplexArrays.java  norm2Sq (LASSQ, :74-140), scal (:159-177)
 *   java.util.SplittableRandom (JDK, not part of the project): the published
 *       SplitMix64 generator (Steele, Lea, Flood, OOPSLA 2014; Vigna splitmix64.c):
 *       state += 0x9e3779b97f4a7c15, Stafford-13 finaliser, nextDouble() =
 *       (nextLong() >>> 11) * 2^-53, nextDouble(b) = nextDouble() * b clamped below b.
 *   java.util.Arrays.binarySearch(double[], double) (JDK): restated in
 *       java_binary_search below, including its doubleToLongBits equality rule.
 *
 * Arithmetic follows the Java scalar paths literally: left-to-right association,
 * no fused multiply-add (compile with -ffp-contract=off).  Index arithmetic is
 * 64-bit so the same code runs past the Java engine's 29-qubit limit.
 * Gate loops carry an optional OpenMP pragma; iterations are independent, so the
 * results do not depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/statecraft_b200.h"

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* SplittableRandom restatement                                              */
/* ------------------------------------------------------------------------ */
typedef struct scx_rng {
  uint64_t seed;
  uint64_t gamma;
} scx_rng;

#define SCX_GOLDEN_GAMMA 0x9e3779b97f4a7c15ULL

static uint64_t scx_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

EXPORT void scx_rng_seed(scx_rng* r, uint64_t seed) {
  r->seed = seed;
  r->gamma = SCX_GOLDEN_GAMMA;
}

EXPORT uint64_t scx_rng_next_long(scx_rng* r) {
  r->seed += r->gamma;
  return scx_mix64(r->seed);
}

EXPORT double scx_rng_next_double(scx_rng* r) {
  return (double)(scx_rng_next_long(r) >> 11) * 0x1.0p-53;
}

EXPORT double scx_rng_next_double_bound(scx_rng* r, double bound) {
  double x = scx_rng_next_double(r);
  x = x * bound;
  if (x >= bound) x = nextafter(bound, -INFINITY);
  return x;
}

/* Fills out[k] with the first `count` nextDouble() values of SplittableRandom(seed). */
EXPORT void scx_uniforms(uint64_t seed, int64_t count, double* out) {
  scx_rng r;
  scx_rng_seed(&r, seed);
  for (int64_t k = 0; k < count; ++k) out[k] = scx_rng_next_double(&r);
}

/* ------------------------------------------------------------------------ */
/* Gate kernels (StatevectorOps scalar paths)                                */
/* ------------------------------------------------------------------------ */
static inline uint64_t insert_zero(uint64_t x, int bit) {
  uint64_t low = x & ((1ULL << bit) - 1ULL);
  return ((x >> bit) << (bit + 1)) | low;
}

EXPORT void scx_apply_single(double* s, int n, int target, const double* g) {
  const double g00r = g[0], g00i = g[1], g01r = g[2], g01i = g[3];
  const double g10r = g[4], g10i = g[5], g11r = g[6], g11i = g[7];
  const uint64_t stride = 1ULL << target;
  const int64_t pairs = (int64_t)(1ULL << (n - 1));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < pairs; ++p) {
    uint64_t idx0 = insert_zero((uint64_t)p, target);
    uint64_t idx1 = idx0 + stride;
    double a0r = s[2 * idx0], a0i = s[2 * idx0 + 1];
    double a1r = s[2 * idx1], a1i = s[2 * idx1 + 1];
    double new0r = g00r * a0r - g00i * a0i + g01r * a1r - g01i * a1i;
    double new0i = g00r * a0i + g00i * a0r + g01r * a1i + g01i * a1r;
    double new1r = g10r * a0r - g10i * a0i + g11r * a1r - g11i * a1i;
    double new1i = g10r * a0i + g10i * a0r + g11r * a1i + g11i * a1r;
    s[2 * idx0] = new0r;
    s[2 * idx0 + 1] = new0i;
    s[2 * idx1] = new1r;
    s[2 * idx1 + 1] = new1i;
  }
}

EXPORT void scx_apply_cnot(double* s, int n, int control, int target) {
  const uint64_t cmask = 1ULL << control, tmask = 1ULL << target;
  const int64_t pairs = (int64_t)(1ULL << (n - 1));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < pairs; ++p) {
    uint64_t idx = insert_zero((uint64_t)p, target);
    if ((idx & cmask) == cmask) {
      uint64_t f = idx | tmask;
      double tr = s[2 * idx], ti = s[2 * idx + 1];
      s[2 * idx] = s[2 * f];
      s[2 * idx + 1] = s[2 * f + 1];
      s[2 * f] = tr;
      s[2 * f + 1] = ti;
    }
  }
}

/* Group layout shared by the two-qubit kernels (StatevectorOps.java:176-188, 991-999). */
typedef struct group_layout {
  int low, high;
  uint64_t off_first, off_second, off_both;
} group_layout;

static group_layout make_layout(int first, int second) {
  group_layout L;
  L.low = first < second ? first : second;
  L.high = first < second ? second : first;
  uint64_t lm = 1ULL << L.low, hm = 1ULL << L.high;
  int first_is_low = (first == L.low);
  L.off_first = first_is_low ? lm : hm;
  L.off_second = first_is_low ? hm : lm;
  L.off_both = lm | hm;
  return L;
}

/* m: 16 complex (re, im) row-major, sc_op layout. */
EXPORT void scx_apply_two(double* s, int n, int first, int second, const double* m) {
  group_layout L = make_layout(first, second);
  double mr[16], mi[16];
  for (int k = 0; k < 16; ++k) {
    mr[k] = m[2 * k];
    mi[k] = m[2 * k + 1];
  }
  const int64_t groups = (int64_t)(1ULL << (n - 2));
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < groups; ++g) {
    uint64_t b = insert_zero(insert_zero((uint64_t)g, L.low), L.high);
    uint64_t i00 = b, i01 = b + L.off_second, i10 = b + L.off_first, i11 = b + L.off_both;
    double a00r = s[2 * i00], a00i = s[2 * i00 + 1];
    double a01r = s[2 * i01], a01i = s[2 * i01 + 1];
    double a10r = s[2 * i10], a10i = s[2 * i10 + 1];
    double a11r = s[2 * i11], a11i = s[2 * i11 + 1];
    double out[8];
    for (int row = 0; row < 4; ++row) {
      const double* r = mr + 4 * row;
      const double* q = mi + 4 * row;
      out[2 * row] = r[0] * a00r - q[0] * a00i + r[1] * a01r - q[1] * a01i + r[2] * a10r -
                     q[2] * a10i + r[3] * a11r - q[3] * a11i;
      out[2 * row + 1] = r[0] * a00i + q[0] * a00r + r[1] * a01i + q[1] * a01r + r[2] * a10i +
                         q[2] * a10r + r[3] * a11i + q[3] * a11r;
    }
    s[2 * i00] = out[0];
    s[2 * i00 + 1] = out[1];
    s[2 * i01] = out[2];
    s[2 * i01 + 1] = out[3];
    s[2 * i10] = out[4];
    s[2 * i10 + 1] = out[5];
    s[2 * i11] = out[6];
    s[2 * i11 + 1] = out[7];
  }
}

/* d: 4 complex (re, im), index 2*bit(first) + bit(second). */
EXPORT void scx_apply_diag2(double* s, int n, int first, int second, const double* d) {
  group_layout L = make_layout(first, second);
  const int64_t groups = (int64_t)(1ULL << (n - 2));
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < groups; ++g) {
    uint64_t b = insert_zero(insert_zero((uint64_t)g, L.low), L.high);
    uint64_t idx[4] = {b, b + L.off_second, b + L.off_first, b + L.off_both};
    for (int k = 0; k < 4; ++k) {
      double ar = s[2 * idx[k]], ai = s[2 * idx[k] + 1];
      double dr = d[2 * k], di = d[2 * k + 1];
      s[2 * idx[k]] = dr * ar - di * ai;
      s[2 * idx[k] + 1] = dr * ai + di * ar;
    }
  }
}

EXPORT void scx_apply_swap(double* s, int n, int first, int second) {
  group_layout L = make_layout(first, second);
  const int64_t groups = (int64_t)(1ULL << (n - 2));
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < groups; ++g) {
    uint64_t b = insert_zero(insert_zero((uint64_t)g, L.low), L.high);
    uint64_t f = b + L.off_first, q = b + L.off_second;
    double fr = s[2 * f], fi = s[2 * f + 1];
    s[2 * f] = s[2 * q];
    s[2 * f + 1] = s[2 * q + 1];
    s[2 * q] = fr;
    s[2 * q + 1] = fi;
  }
}

EXPORT void scx_apply_multi(double* s, int n, int target, uint64_t cmask, const double* g) {
  const double g00r = g[0], g00i = g[1], g01r = g[2], g01i = g[3];
  const double g10r = g[4], g10i = g[5], g11r = g[6], g11i = g[7];
  const uint64_t stride = 1ULL << target;
  const int64_t pairs = (int64_t)(1ULL << (n - 1));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < pairs; ++p) {
    uint64_t idx0 = insert_zero((uint64_t)p, target);
    if ((idx0 & cmask) != cmask) continue;
    uint64_t idx1 = idx0 + stride;
    double a0r = s[2 * idx0], a0i = s[2 * idx0 + 1];
    double a1r = s[2 * idx1], a1i = s[2 * idx1 + 1];
    double new0r = g00r * a0r - g00i * a0i + g01r * a1r - g01i * a1i;
    double new0i = g00r * a0i + g00i * a0r + g01r * a1i + g01i * a1r;
    double new1r = g10r * a0r - g10i * a0i + g11r * a1r - g11i * a1i;
    double new1i = g10r * a0i + g10i * a0r + g11r * a1i + g11i * a1r;
    s[2 * idx0] = new0r;
    s[2 * idx0 + 1] = new0i;
    s[2 * idx1] = new1r;
    s[2 * idx1 + 1] = new1i;
  }
}

/* Matrices of the parameterised rotations (OpenQasmCircuitParser.java:650-670). */
EXPORT void scx_rotation_matrix(int kind, double a, double* g) {
  double half = a / 2.0;
  double c = cos(half), sn = sin(half);
  memset(g, 0, 8 * sizeof(double));
  if (kind == SC_OP_RX) {
    g[0] = c; g[3] = -sn; g[5] = -sn; g[6] = c;
  } else if (kind == SC_OP_RY) {
    g[0] = c; g[2] = -sn; g[4] = sn; g[6] = c;
  } else { /* RZ: diag(cis(-a/2), cis(a/2)) */
    g[0] = cos(-half); g[1] = sin(-half); g[6] = cos(half); g[7] = sin(half);
  }
}

/* RZZ(a) = exp(-i a/2 Z Z) = diag(cis(-a/2), cis(a/2), cis(a/2), cis(-a/2)). */
EXPORT void scx_rzz_diagonal(double a, double* d) {
  double h = a / 2.0;
  d[0] = cos(-h); d[1] = sin(-h);
  d[2] = cos(h); d[3] = sin(h);
  d[4] = cos(h); d[5] = sin(h);
  d[6] = cos(-h); d[7] = sin(-h);
}

/* ------------------------------------------------------------------------ */
/* LASSQ norm and scal (ComplexArrays.java:74-140, 159-177)                  */
/* ------------------------------------------------------------------------ */
EXPORT double scx_norm2sq(const double* a, int64_t count) {
  double scale = 0.0, ssq = 1.0;
  for (int64_t k = 0; k < count; ++k) {
    double re = a[2 * k], im = a[2 * k + 1];
    if (isnan(re) || isnan(im)) return NAN;
    if (isinf(re) || isinf(im)) return INFINITY;
    double ar = fabs(re);
    if (ar != 0.0) {
      if (scale < ar) {
        double r = scale / ar;
        ssq = 1.0 + ssq * r * r;
        scale = ar;
      } else if (scale != 0.0) {
        double r = ar / scale;
        ssq += r * r;
      } else {
        scale = ar;
      }
    }
    double ai = fabs(im);
    if (ai != 0.0) {
      if (scale < ai) {
        double r = scale / ai;
        ssq = 1.0 + ssq * r * r;
        scale = ai;
      } else if (scale != 0.0) {
        double r = ai / scale;
        ssq += r * r;
      } else {
        scale = ai;
      }
    }
  }
  return scale == 0.0 ? 0.0 : (scale * scale) * ssq;
}

static void scal_real(double* x, int64_t count, double alpha) {
  const double alpha_im = 0.0;
  for (int64_t k = 0; k < count; ++k) {
    double xr = x[2 * k], xi = x[2 * k + 1];
    double rr = alpha * xr - alpha_im * xi;
    double ri = alpha * xi + alpha_im * xr;
    x[2 * k] = rr;
    x[2 * k + 1] = ri;
  }
}

/* ------------------------------------------------------------------------ */
/* Kraus trajectory step (StatevectorEngine.java:463-600)                    */
/* ------------------------------------------------------------------------ */
#define SCX_MIN_KRAUS_WEIGHT 1e-15

static double branch_weight(const double* s, int n, int target, const double* k) {
  const uint64_t tmask = 1ULL << target;
  const uint64_t dim = 1ULL << n;
  double weight = 0.0;
  for (uint64_t basis = 0; basis < dim; ++basis) {
    if (basis & tmask) continue;
    double in[4] = {s[2 * basis], s[2 * basis + 1], s[2 * (basis | tmask)],
                    s[2 * (basis | tmask) + 1]};
    double out[4];
    for (int row = 0; row < 2; ++row) {
      double sr = 0.0, si = 0.0;
      for (int col = 0; col < 2; ++col) {
        double cr = k[4 * row + 2 * col], ci = k[4 * row + 2 * col + 1];
        double ar = in[2 * col], ai = in[2 * col + 1];
        sr += cr * ar - ci * ai;
        si += cr * ai + ci * ar;
      }
      out[2 * row] = sr;
      out[2 * row + 1] = si;
    }
    double nsq = 0.0;
    for (int q = 0; q < 4; q += 2) nsq += out[q] * out[q] + out[q + 1] * out[q + 1];
    weight += nsq;
  }
  return weight;
}

static int sample_weighted_index(const double* w, int count, double value) {
  double cumulative = 0.0;
  for (int k = 0; k < count; ++k) {
    cumulative += w[k];
    if (value < cumulative) return k;
  }
  return count - 1;
}

/* One channel application on one target; returns the chosen Kraus index or a
 * negative status. */
EXPORT int scx_apply_channel(double* s, int n, const sc_channel* ch, scx_rng* rng,
                             double* weights_out) {
  double w[SC_MAX_KRAUS];
  double total = 0.0;
  for (int k = 0; k < ch->n_kraus; ++k) {
    double bw = branch_weight(s, n, ch->target, ch->kraus[k]);
    if (!isfinite(bw) || bw < 0.0) return SC_ESTATE;
    w[k] = bw;
    total += bw;
  }
  if (!isfinite(total) || total <= SCX_MIN_KRAUS_WEIGHT) return SC_ESTATE;
  if (weights_out)
    for (int k = 0; k < ch->n_kraus; ++k) weights_out[k] = w[k];
  int idx = sample_weighted_index(w, ch->n_kraus, scx_rng_next_double_bound(rng, total));
  scx_apply_single(s, n, ch->target, ch->kraus[idx]);
  const int64_t dim = (int64_t)(1ULL << n);
  double nsq = scx_norm2sq(s, dim);
  if (!isfinite(nsq) || nsq == 0.0) return SC_ESTATE;
  if (fabs(nsq - 1.0) > 1e-12) scal_real(s, dim, 1.0 / sqrt(nsq));
  return idx;
}

/* ------------------------------------------------------------------------ */
/* simulate() op loop                                                        */
/* ------------------------------------------------------------------------ */
static int is_unitary_kind(int kind) {
  return kind == SC_OP_SINGLE || kind == SC_OP_CNOT || kind == SC_OP_TWO ||
         kind == SC_OP_DIAG2 || kind == SC_OP_SWAP || kind == SC_OP_MULTI || kind == SC_OP_RX ||
         kind == SC_OP_RY || kind == SC_OP_RZ || kind == SC_OP_RZZ;
}

static double op_angle(const sc_op* op, const double* params, int64_t n_params) {
  if (op->param >= 0 && params && op->param < n_params) return params[op->param];
  return op->m[0];
}

/* Applies one unitary op. */
EXPORT int scx_apply_op(double* s, int n, const sc_op* op, const double* params,
                        int64_t n_params) {
  double g[8], d[8];
  switch (op->kind) {
    case SC_OP_SINGLE: scx_apply_single(s, n, op->q0, op->m); return SC_OK;
    case SC_OP_CNOT: scx_apply_cnot(s, n, op->q0, op->q1); return SC_OK;
    case SC_OP_TWO: scx_apply_two(s, n, op->q0, op->q1, op->m); return SC_OK;
    case SC_OP_DIAG2: scx_apply_diag2(s, n, op->q0, op->q1, op->m); return SC_OK;
    case SC_OP_SWAP: scx_apply_swap(s, n, op->q0, op->q1); return SC_OK;
    case SC_OP_MULTI: scx_apply_multi(s, n, op->q0, op->mask, op->m); return SC_OK;
    case SC_OP_RX:
    case SC_OP_RY:
    case SC_OP_RZ:
      scx_rotation_matrix(op->kind, op_angle(op, params, n_params), g);
      scx_apply_single(s, n, op->q0, g);
      return SC_OK;
    case SC_OP_RZZ:
      scx_rzz_diagonal(op_angle(op, params, n_params), d);
      scx_apply_diag2(s, n, op->q0, op->q1, d);
      return SC_OK;
    default: return SC_EINVAL;
  }
}

/* Runs ops on `s` (already initialised).  Channels must be sorted by after_op.
 * chosen_out (nullable, n_ch entries) receives the sampled Kraus index per channel.
 * Returns SC_OK or a status mirroring the exception the Java engine raises. */
EXPORT int scx_run(double* s, int n, const sc_op* ops, int64_t n_ops, const double* params,
                   int64_t n_params, const sc_channel* ch, int64_t n_ch, uint64_t noise_seed,
                   int32_t* chosen_out) {
  scx_rng rng;
  scx_rng_seed(&rng, noise_seed);
  int64_t next = 0;
  int measured = 0;
  for (int64_t i = 0; i < n_ops; ++i) {
    const sc_op* op = &ops[i];
    if (op->kind == SC_OP_MEASURE) {
      measured = 1;
      continue;
    }
    if (!is_unitary_kind(op->kind)) return SC_EINVAL;
    if (measured) return SC_EUNSUPPORTED;
    int rc = scx_apply_op(s, n, op, params, n_params);
    if (rc != SC_OK) return rc;
    while (next < n_ch && ch[next].after_op == i) {
      if (ch[next].target < 0 || ch[next].target >= n) return SC_EINVAL;
      int idx = scx_apply_channel(s, n, &ch[next], &rng, NULL);
      if (idx < 0) return idx;
      if (chosen_out) chosen_out[next] = idx;
      ++next;
    }
  }
  return SC_OK;
}

/* ------------------------------------------------------------------------ */
/* Measurement (StatevectorEngine.java:274-338)                              */
/* ------------------------------------------------------------------------ */
EXPORT void scx_probabilities(const double* s, int n, const int32_t* qubits, int m,
                              double* probs) {
  const uint64_t dim = 1ULL << n;
  memset(probs, 0, sizeof(double) * ((size_t)1 << m));
  uint64_t covered = 0;
  for (int bit = 0; bit < m; ++bit) covered |= 1ULL << qubits[bit];
  if (m == n && covered == dim - 1) {
    /* every qubit measured once: each outcome receives exactly one basis state's p, so the
     * loop has no accumulation order and runs in parallel with identical results */
#pragma omp parallel for schedule(static)
    for (int64_t basis = 0; basis < (int64_t)dim; ++basis) {
      double ar = s[2 * basis], ai = s[2 * basis + 1];
      double p = (ar * ar) + (ai * ai);
      if (p == 0.0) continue;
      uint64_t outcome = 0;
      for (int bit = 0; bit < m; ++bit)
        if (((uint64_t)basis >> qubits[bit]) & 1ULL) outcome |= (1ULL << bit);
      probs[outcome] = p;
    }
    return;
  }
  for (uint64_t basis = 0; basis < dim; ++basis) {
    double ar = s[2 * basis], ai = s[2 * basis + 1];
    double p = (ar * ar) + (ai * ai);
    if (p == 0.0) continue;
    uint64_t outcome = 0;
    for (int bit = 0; bit < m; ++bit)
      if ((basis >> qubits[bit]) & 1ULL) outcome |= (1ULL << bit);
    probs[outcome] += p;
  }
}

EXPORT int scx_normalize(double* probs, int64_t len) {
  double sum = 0.0;
  for (int64_t k = 0; k < len; ++k) sum += probs[k];
  if (sum == 0.0) return SC_ESTATE;
  if (fabs(sum - 1.0) > 1e-12) {
    double scale = 1.0 / sum;
    for (int64_t k = 0; k < len; ++k) probs[k] *= scale;
  }
  return SC_OK;
}

EXPORT void scx_cumulative(const double* probs, int64_t len, double* cdf) {
  double running = 0.0;
  for (int64_t k = 0; k < len; ++k) {
    running += probs[k];
    cdf[k] = running;
  }
  cdf[len - 1] = 1.0;
}

static int64_t double_bits(double x) {
  int64_t b;
  if (isnan(x)) return 0x7ff8000000000000LL; /* doubleToLongBits canonical NaN */
  memcpy(&b, &x, sizeof b);
  return b;
}

/* java.util.Arrays.binarySearch(double[], double) */
static int64_t java_binary_search(const double* a, int64_t len, double key) {
  int64_t low = 0, high = len - 1;
  while (low <= high) {
    int64_t mid = (int64_t)(((uint64_t)low + (uint64_t)high) >> 1);
    double midv = a[mid];
    if (midv < key) {
      low = mid + 1;
    } else if (midv > key) {
      high = mid - 1;
    } else {
      int64_t mb = double_bits(midv), kb = double_bits(key);
      if (mb == kb) return mid;
      if (mb < kb) low = mid + 1;
      else high = mid - 1;
    }
  }
  return -(low + 1);
}

EXPORT int64_t scx_sample_outcome(const double* cdf, int64_t len, double value) {
  if (value >= 1.0) return len - 1;
  int64_t index = java_binary_search(cdf, len, value);
  if (index >= 0) {
    while (index > 0 && cdf[index - 1] >= value) index--;
    return index;
  }
  return -index - 1;
}

/* Full measurement: probabilities -> normalize -> cumulative -> per-shot search.
 * uniforms nullable: then SplittableRandom(seed).nextDouble() per shot. */
EXPORT int scx_sample(const double* s, int n, const int32_t* qubits, int m, int64_t shots,
                      uint64_t seed, const double* uniforms, int32_t* out) {
  const int64_t len = (int64_t)1 << m;
  double* probs = (double*)malloc(sizeof(double) * (size_t)len);
  double* cdf = (double*)malloc(sizeof(double) * (size_t)len);
  if (!probs || !cdf) {
    free(probs);
    free(cdf);
    return SC_ENOMEM;
  }
  scx_probabilities(s, n, qubits, m, probs);
  int rc = scx_normalize(probs, len);
  if (rc == SC_OK) {
    scx_cumulative(probs, len, cdf);
    scx_rng rng;
    scx_rng_seed(&rng, seed);
    for (int64_t k = 0; k < shots; ++k) {
      double u = uniforms ? uniforms[k] : scx_rng_next_double(&rng);
      out[k] = (int32_t)scx_sample_outcome(cdf, len, u);
    }
  }
  free(probs);
  free(cdf);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Pauli-sum expectation (addition: no counterpart in the reference)         */
/* ------------------------------------------------------------------------ */
/* Term acts as X on xmask bits, Z on zmask bits, Y (= i X Z) where both are set.
 * (P psi)_i = i^{ny} (-1)^{popcount(z & (i ^ x))} psi_{i ^ x}. */
EXPORT double scx_expect_pauli(const double* s, int n, int32_t n_terms, const uint64_t* xm,
                               const uint64_t* zm, const double* coeffs) {
  const uint64_t dim = 1ULL << n;
  double total = 0.0;
  for (int32_t t = 0; t < n_terms; ++t) {
    uint64_t x = xm[t], z = zm[t];
    int ny = __builtin_popcountll(x & z) & 3;
    double acc_r = 0.0, acc_i = 0.0;
    for (uint64_t i = 0; i < dim; ++i) {
      uint64_t j = i ^ x;
      double sign = (__builtin_popcountll(z & j) & 1) ? -1.0 : 1.0;
      double pr = sign * s[2 * j], pi = sign * s[2 * j + 1];
      /* multiply by i^ny */
      for (int k = 0; k < ny; ++k) {
        double t0 = -pi;
        pi = pr;
        pr = t0;
      }
      /* conj(psi_i) * (P psi)_i */
      acc_r += s[2 * i] * pr + s[2 * i + 1] * pi;
      acc_i += s[2 * i] * pi - s[2 * i + 1] * pr;
    }
    total += coeffs[t] * acc_r;
  }
  return total;
}
