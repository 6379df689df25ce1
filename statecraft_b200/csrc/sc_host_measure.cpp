// Host side of measurement and expectation values: validation mirroring
// StatevectorEngine.performMeasurement (StatevectorEngine.java:229-312) and the
// scratch-buffer layout of the device sampler.
#include <cmath>
#include <cstring>

#include "sc_ctx.h"

namespace sc {

namespace {

int validate_measured(const int32_t* qubits, int32_t m, int n, uint64_t* mmask) {
  if (m <= 0 || !qubits) return fail(SC_ESTATE, "No qubits available for measurement");
  uint64_t mask = 0;
  for (int32_t k = 0; k < m; ++k) {
    const int q = qubits[k];
    if (q < 0 || q >= n) return fail(SC_EINVAL, "measurement qubit out of range: %d", q);
    if (k > 0 && q <= qubits[k - 1])
      return fail(SC_EINVAL, "measured qubits must be ascending and distinct (got %d after %d)", q,
                  qubits[k - 1]);
    mask |= 1ULL << q;
  }
  *mmask = mask;
  return SC_OK;
}

}  // namespace

int Ctx::sample(const int32_t* qubits, int32_t m, int64_t shots, uint64_t seed,
                const double* uniforms, int32_t* outcomes) {
  if (!state_valid) return fail(SC_ESTATE, "no state: sc_run has not completed");
  uint64_t mmask = 0;
  int rc = validate_measured(qubits, m, n, &mmask);
  if (rc != SC_OK) return rc;
  if (shots <= 0) return fail(SC_EINVAL, "shots must be positive");
  if (!outcomes) return fail(SC_EINVAL, "outcomes buffer is null");
  if (uniforms)
    for (int64_t k = 0; k < shots; ++k)
      if (!std::isfinite(uniforms[k])) return fail(SC_EINVAL, "uniform %lld is not finite", (long long)k);

  const bool direct = (m == n);
  const uint64_t len = 1ULL << m;
  const double dim = std::ldexp(1.0, n);
  const double amp_bytes = (cfg.dtype == SC_C64) ? 8.0 : 16.0;
  double* probs = nullptr;
  if (!direct) {
    if ((rc = reserve(buf_probs, sizeof(double) * len, "marginal probabilities")) != SC_OK) return rc;
    const uint64_t rest = 1ULL << (n - m);
    size_t marg_elems = 1;
    if (rest > 64) marg_elems = (size_t)len * (size_t)((rest + kSampleChunk - 1) / kSampleChunk);
    if ((rc = reserve(buf_marg, sizeof(double) * marg_elems, "marginal partials")) != SC_OK) return rc;
    probs = static_cast<double*>(buf_probs.p);
    mark_begin(KC_PROB, dim * amp_bytes + 8.0 * (double)len, rest > 64 ? 2 : 1);
    cudaError_t e = launch_marginal(cfg.dtype, state.p, n, mmask, m, probs,
                                    static_cast<double*>(buf_marg.p), marg_elems, sm_count, stream);
    mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "marginal kernel");
  }
  const uint64_t chunks = sample_chunks(len);
  const size_t off_prefix = sizeof(double) * chunks;
  const size_t off_start = 2 * off_prefix;
  const size_t off_tf = 3 * off_prefix;
  const size_t off_scalars = off_tf + sizeof(ChunkTf) * chunks;
  const size_t off_uniforms = off_scalars + 64;
  const size_t off_outcomes = off_uniforms + (uniforms ? sizeof(double) * (size_t)shots : 0);
  const size_t total = off_outcomes + sizeof(int32_t) * (size_t)shots + 16;
  if ((rc = reserve(buf_sample, total, "sampler scratch")) != SC_OK) return rc;
  char* base = static_cast<char*>(buf_sample.p);
  SampleArgs a;
  a.chunk_sums = reinterpret_cast<double*>(base);
  a.chunk_prefix = reinterpret_cast<double*>(base + off_prefix);
  a.chunk_start = reinterpret_cast<double*>(base + off_start);
  a.chunk_tf = reinterpret_cast<ChunkTf*>(base + off_tf);
  a.scalars = reinterpret_cast<SampleScalars*>(base + off_scalars);
  a.uniforms = uniforms ? reinterpret_cast<const double*>(base + off_uniforms) : nullptr;
  a.seed = seed;
  a.shots = shots;
  a.outcomes = reinterpret_cast<int32_t*>(base + off_outcomes);
  a.sm_count = sm_count;
  cudaError_t e;
  if (uniforms) {
    e = cudaMemcpyAsync(base + off_uniforms, uniforms, sizeof(double) * (size_t)shots,
                        cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return fail_cuda(e, "uniform upload");
  }
  mark_begin(KC_SAMPLE, (direct ? dim * amp_bytes : 8.0 * (double)len), kSampleKernels);
  e = launch_sample(cfg.dtype, state.p, probs, len, a, stream);
  mark_end();
  if (e != cudaSuccess) return fail_cuda(e, "sampling kernels");
  SampleScalars sc_host;
  if ((e = cudaMemcpyAsync(&sc_host, a.scalars, sizeof sc_host, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(outcomes, a.outcomes, sizeof(int32_t) * (size_t)shots,
                           cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return fail_cuda(e, "outcome download");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "sc_sample");
  collect_timing();
  if (sc_host.status != 0) return fail(SC_ESTATE, "State collapsed to zero probability amplitudes");
  return SC_OK;
}

int Ctx::probabilities(const int32_t* qubits, int32_t m, double* out) {
  if (!state_valid) return fail(SC_ESTATE, "no state: sc_run has not completed");
  uint64_t mmask = 0;
  int rc = validate_measured(qubits, m, n, &mmask);
  if (rc != SC_OK) return rc;
  if (!out) return fail(SC_EINVAL, "output buffer is null");
  const uint64_t len = 1ULL << m;
  if ((rc = reserve(buf_probs, sizeof(double) * len, "marginal probabilities")) != SC_OK) return rc;
  const uint64_t rest = 1ULL << (n - m);
  size_t marg_elems = 1;
  if (rest > 64) marg_elems = (size_t)len * (size_t)((rest + kSampleChunk - 1) / kSampleChunk);
  if ((rc = reserve(buf_marg, sizeof(double) * marg_elems, "marginal partials")) != SC_OK) return rc;
  cudaError_t e = launch_marginal(cfg.dtype, state.p, n, mmask, m, static_cast<double*>(buf_probs.p),
                                  static_cast<double*>(buf_marg.p), marg_elems, sm_count, stream);
  if (e != cudaSuccess) return fail_cuda(e, "marginal kernel");
  if ((e = cudaMemcpyAsync(out, buf_probs.p, sizeof(double) * len, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return fail_cuda(e, "probability download");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "sc_probabilities");
  // normalize (StatevectorEngine.java:298-312)
  double sum = 0.0;
  for (uint64_t k = 0; k < len; ++k) sum += out[k];
  if (sum == 0.0) return fail(SC_ESTATE, "State collapsed to zero probability amplitudes");
  if (std::fabs(sum - 1.0) > 1e-12) {
    const double scale = 1.0 / sum;
    for (uint64_t k = 0; k < len; ++k) out[k] *= scale;
  }
  return SC_OK;
}

int Ctx::pauli_terms(int32_t n_terms, const uint64_t* xmask, const uint64_t* zmask,
                     std::vector<double>& terms) {
  if (n_terms < 0 || (n_terms > 0 && (!xmask || !zmask)))
    return fail(SC_EINVAL, "invalid Pauli term arrays");
  const uint64_t full = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
  for (int32_t t = 0; t < n_terms; ++t)
    if ((xmask[t] | zmask[t]) & ~full) return fail(SC_EINVAL, "Pauli term %d acts outside the register", t);
  terms.assign(n_terms, 0.0);
  if (n_terms == 0) return SC_OK;
  const int cols = pauli_partial_cols(n, sm_count);
  const size_t elems = (size_t)cols * n_terms + n_terms;
  int rc = reserve(buf_expect, sizeof(double) * elems, "expectation partials");
  if (rc != SC_OK) return rc;
  double* part = static_cast<double*>(buf_expect.p);
  double* out = part + (size_t)cols * n_terms;
  const double amp_bytes = (cfg.dtype == SC_C64) ? 8.0 : 16.0;
  mark_begin(KC_EXPECT, 2.0 * std::ldexp(1.0, n) * amp_bytes * n_terms, n_terms + 1);
  cudaError_t e = launch_pauli_terms(cfg.dtype, state.p, n, n_terms, xmask, zmask, part,
                                     (size_t)cols * n_terms, out, sm_count, stream);
  mark_end();
  if (e != cudaSuccess) return fail_cuda(e, "expectation kernels");
  if ((e = cudaMemcpyAsync(terms.data(), out, sizeof(double) * n_terms, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return fail_cuda(e, "expectation download");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "expectation");
  collect_timing();
  return SC_OK;
}

}  // namespace sc
