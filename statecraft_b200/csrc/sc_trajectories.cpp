// Batched noisy trajectories (addition; the reference runs one trajectory per
// StatevectorEngine.simulate call, StatevectorEngine.java:371-600).
//
// Every noise record must be a Pauli mixture: each Kraus operator K_k = c_k P_k
// with P_k in {I, X, Y, Z} (depolarizing, bit / phase flip, Pauli channels).  Then
// the branch weight the reference computes, ||K_k psi||^2, is |c_k|^2 for the
// normalised state, so trajectory t's branch choices are fixed by its
// SplittableRandom(noise_seed + t) alone: record j takes the j-th nextDouble(total)
// draw and the reference's cumulative-weight rule (sampleWeightedIndex).  The
// host draws every choice up front; the device runs ONE fused plan for all
// trajectories, with a Pauli slot after each op that carries noise, each
// trajectory reading its Pauli from a choice table.  Each sweep is one launch
// over all trajectories' states, stored back to back in HBM.
#include <cmath>
#include <cstring>
#include <vector>

#include "sc_ctx.h"
#include "sc_rng.h"

namespace sc {

namespace {

// Kraus matrix k (2x2 row-major complex) as c * P; returns the Pauli code
// (0 I, 1 X, 2 Y, 3 Z) and |c|^2, or -1 if it is not a scaled Pauli.
int pauli_of(const double* k, double* weight) {
  auto zero = [](double r, double i) { return r == 0.0 && i == 0.0; };
  const double a_r = k[0], a_i = k[1], b_r = k[2], b_i = k[3];
  const double c_r = k[4], c_i = k[5], d_r = k[6], d_i = k[7];
  if (zero(b_r, b_i) && zero(c_r, c_i)) {
    if (a_r == d_r && a_i == d_i) {
      *weight = a_r * a_r + a_i * a_i;
      return 0;
    }
    if (a_r == -d_r && a_i == -d_i) {
      *weight = a_r * a_r + a_i * a_i;
      return 3;
    }
    return -1;
  }
  if (zero(a_r, a_i) && zero(d_r, d_i)) {
    if (b_r == c_r && b_i == c_i) {
      *weight = b_r * b_r + b_i * b_i;
      return 1;
    }
    if (b_r == -c_r && b_i == -c_i) {  // Y = [[0, -i], [i, 0]] scaled by c = i * k01
      *weight = b_r * b_r + b_i * b_i;
      return 2;
    }
  }
  return -1;
}

// java.util.SplittableRandom(seed): the k-th nextDouble(bound)
double next_double_bound(uint64_t seed, uint64_t k, double bound) {
  double x = splitmix_double(seed, k) * bound;
  if (x >= bound) x = std::nextafter(bound, -INFINITY);
  return x;
}

int weighted_index(const double* w, int count, double value) {
  double cumulative = 0.0;
  for (int k = 0; k < count; ++k) {
    cumulative += w[k];
    if (value < cumulative) return k;
  }
  return count - 1;
}

constexpr double kMinKrausWeight = 1e-15;

}  // namespace

}  // namespace sc

using namespace sc;

extern "C" {

int32_t sc_trajectories(void* p, int32_t n, const sc_op* ops, int64_t n_ops,
                        const sc_channel* channels, int64_t n_channels, int64_t n_traj,
                        uint64_t noise_seed, int64_t shots, uint64_t measure_seed,
                        int32_t* outcomes, int32_t* choices, double* states) {
  int rc = check_context(p);
  if (rc != SC_OK) return rc;
  Ctx* c = static_cast<Ctx*>(p);
  if (n_traj < 1 || n_traj > 65535) return fail(SC_EINVAL, "trajectory count must be in 1..65535");
  if (shots < 0 || (shots > 0 && !outcomes)) return fail(SC_EINVAL, "invalid shots / outcome buffer");
  if (n_channels < 0 || (n_channels > 0 && !channels)) return fail(SC_EINVAL, "invalid noise records");
  if ((rc = validate_circuit(n, ops, n_ops, c->max_qubits)) != SC_OK) return rc;
  std::vector<sc_channel> ch(channels, channels + n_channels);
  if ((rc = validate_noise(ch, ops, n_ops, n)) != SC_OK) return rc;

  // Pauli decomposition of every record
  std::vector<double> weight((size_t)n_channels * SC_MAX_KRAUS, 0.0);
  std::vector<uint8_t> code((size_t)n_channels * SC_MAX_KRAUS, 0);
  for (int64_t j = 0; j < n_channels; ++j) {
    double total = 0.0;
    for (int k = 0; k < ch[j].n_kraus; ++k) {
      double w = 0.0;
      const int pc = pauli_of(ch[j].kraus[k], &w);
      if (pc < 0)
        return fail(SC_EUNSUPPORTED,
                    "noise record %lld: Kraus operator %d is not a scaled Pauli; trajectory "
                    "batches take Pauli-mixture channels", (long long)j, k);
      weight[j * SC_MAX_KRAUS + k] = w;
      code[j * SC_MAX_KRAUS + k] = (uint8_t)pc;
      total += w;
    }
    if (!std::isfinite(total) || total <= kMinKrausWeight)
      return fail(SC_ESTATE, "noise record %lld: invalid Kraus branch weights", (long long)j);
  }

  // one gate list for every trajectory: ops with a Pauli slot after each noise record
  std::vector<PGate> gates;
  int64_t next = 0;
  for (int64_t i = 0; i < n_ops; ++i) {
    PGate g;
    bool produced = false;
    if (!normalise_op(ops[i], nullptr, 0, &g, &produced))
      return fail(SC_EINVAL, "op %lld: cannot normalise", (long long)i);
    if (produced) {
      g.op_index = i;
      gates.push_back(g);
    }
    while (next < n_channels && ch[next].after_op == i) {
      PGate s;
      std::memset(&s, 0, sizeof s);
      s.kind = PK_PAULI;
      s.q0 = ch[next].target;
      s.q1 = (int32_t)next;
      s.op_index = i;
      gates.push_back(s);
      ++next;
    }
  }
  PlanParams pp = c->plan_params();
  pp.relayout = false;  // the batch is planned once; no layout to restore
  Plan plan = plan_sweeps(gates, n, pp);
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");

  // branch choices, drawn as the reference draws them
  const size_t n_ch = (size_t)n_channels;
  std::vector<uint8_t> paulis(std::max<size_t>(1, (size_t)n_traj * n_ch), 0);
  for (int64_t t = 0; t < n_traj; ++t) {
    const uint64_t seed = noise_seed + (uint64_t)t;
    for (size_t j = 0; j < n_ch; ++j) {
      const double* w = &weight[j * SC_MAX_KRAUS];
      double total = 0.0;
      for (int k = 0; k < ch[j].n_kraus; ++k) total += w[k];
      const int idx = weighted_index(w, ch[j].n_kraus, next_double_bound(seed, j, total));
      paulis[(size_t)t * n_ch + j] = code[j * SC_MAX_KRAUS + idx];
      if (choices) choices[(size_t)t * n_ch + j] = idx;
    }
  }

  // device buffers: states | Pauli table, sampling scratch, outcomes
  const size_t amp = c->cfg.dtype == SC_C64 ? 8 : 16;
  const uint64_t len = 1ULL << n;
  const size_t state_bytes = amp * len * (size_t)n_traj;
  const uint64_t chunks = sample_chunks(len);
  const size_t off_codes = 0;
  const size_t off_sums = (paulis.size() + 255) & ~(size_t)255;
  const size_t off_prefix = off_sums + sizeof(double) * chunks * (size_t)n_traj;
  const size_t off_start = off_prefix + sizeof(double) * chunks * (size_t)n_traj;
  const size_t off_tf = off_start + sizeof(double) * chunks * (size_t)n_traj;
  const size_t off_scalars = off_tf + sizeof(ChunkTf) * chunks * (size_t)n_traj;
  const size_t off_out = off_scalars + sizeof(SampleScalars) * (size_t)n_traj;
  const size_t aux_bytes = off_out + sizeof(int32_t) * (size_t)std::max<int64_t>(1, shots * n_traj);
  if ((rc = c->reserve(c->buf_traj_states, state_bytes, "trajectory states")) != SC_OK) return rc;
  if ((rc = c->reserve(c->buf_traj_aux, aux_bytes, "trajectory scratch")) != SC_OK) return rc;
  if ((rc = c->reserve(c->buf_err, 16, "error flag")) != SC_OK) return rc;
  char* aux = static_cast<char*>(c->buf_traj_aux.p);
  cudaStream_t s = c->stream;
  cudaError_t e = cudaMemsetAsync(c->buf_err.p, 0, 16, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(aux + off_codes, paulis.data(), paulis.size(), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail_cuda(e, "trajectory set-up");

  const double dim = std::ldexp(1.0, n);
  c->mark_begin(KC_INIT, dim * (double)amp * (double)n_traj);
  e = launch_init_batch(c->cfg.dtype, c->buf_traj_states.p, n, n_traj, s);
  c->mark_end();
  if (e != cudaSuccess) return fail_cuda(e, "trajectory init");
  for (size_t k = 0; k < plan.sweeps.size(); ++k) {
    c->mark_begin(KC_SWEEP, 2.0 * dim * (double)amp * (double)n_traj);
    e = launch_sweep_batch(c->cfg.dtype, c->buf_traj_states.p, n, n_traj, plan, k,
                           reinterpret_cast<const uint8_t*>(aux + off_codes), (int)n_ch,
                           static_cast<int*>(c->buf_err.p), c->sm_count, s);
    c->mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "trajectory sweep");
  }
  std::vector<SampleScalars> scal((size_t)n_traj);
  if (shots > 0) {
    SampleArgs a;
    a.chunk_sums = reinterpret_cast<double*>(aux + off_sums);
    a.chunk_prefix = reinterpret_cast<double*>(aux + off_prefix);
    a.chunk_start = reinterpret_cast<double*>(aux + off_start);
    a.chunk_tf = reinterpret_cast<ChunkTf*>(aux + off_tf);
    a.scalars = reinterpret_cast<SampleScalars*>(aux + off_scalars);
    a.uniforms = nullptr;
    a.seed = measure_seed;
    a.shots = shots;
    a.outcomes = reinterpret_cast<int32_t*>(aux + off_out);
    a.sm_count = c->sm_count;
    c->mark_begin(KC_SAMPLE, dim * (double)amp * (double)n_traj, 3);
    e = launch_sample_batch(c->cfg.dtype, c->buf_traj_states.p, len, n_traj, a, s);
    c->mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "trajectory sampling");
    e = cudaMemcpyAsync(scal.data(), a.scalars, sizeof(SampleScalars) * scal.size(),
                        cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(outcomes, a.outcomes, sizeof(int32_t) * (size_t)(shots * n_traj),
                          cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return fail_cuda(e, "outcome download");
  }
  if (states) {
    // host copy of every final state as interleaved doubles (c64 widened first,
    // in the sampling scratch of the single-run path)
    const size_t out_bytes = 16 * len * (size_t)n_traj;
    if (c->cfg.dtype == SC_C64) {
      if ((rc = c->reserve(c->buf_convert, out_bytes, "state staging")) != SC_OK) return rc;
      e = launch_convert_out(c->cfg.dtype, c->buf_traj_states.p,
                             static_cast<double*>(c->buf_convert.p), (int64_t)(len * n_traj), s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(states, c->buf_convert.p, out_bytes, cudaMemcpyDeviceToHost, s);
    } else {
      e = cudaMemcpyAsync(states, c->buf_traj_states.p, out_bytes, cudaMemcpyDeviceToHost, s);
    }
    if (e != cudaSuccess) return fail_cuda(e, "state download");
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail_cuda(e, "sc_trajectories");
  c->collect_timing();
  int err_flag = 0;
  if ((e = cudaMemcpy(&err_flag, c->buf_err.p, sizeof err_flag, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "error flag");
  if (err_flag) return fail(SC_ETIMEOUT, "sweep kernel timed out waiting for a bulk copy");
  for (int64_t t = 0; t < (shots > 0 ? n_traj : 0); ++t)
    if (scal[t].status != 0)
      return fail(SC_ESTATE, "trajectory %lld: state collapsed to zero probability amplitudes",
                  (long long)t);
  c->plan_sweeps_count = (int64_t)plan.sweeps.size();
  c->plan_gates = plan.n_gates;
  c->plan_stages = (int64_t)plan.stages.size();
  return SC_OK;
}

}  // extern "C"
