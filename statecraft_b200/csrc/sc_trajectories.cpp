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
#include <algorithm>
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

// One piece of the batch between two Kraus points: the fused plan of its gates, Pauli
// slots and the matrix records of earlier Kraus points, then (kraus >= 0) the noise
// record whose branch weights depend on the state, weighed and drawn on the device
// (Kraus point number kp; with pend_kp >= 0, the matrix of that earlier point on
// qubit pend_q is not applied yet and is applied while weighing).
struct Segment {
  Plan plan;
  int64_t kraus = -1, kp = -1, pend_kp = -1;
  int pend_q = -1;
};

// Offsets in the trajectory scratch buffer
struct AuxLayout {
  size_t codes, seeds, sums, prefix, start, tf, scalars, out, partial, mats, kchoice, status, bytes;
};

AuxLayout aux_layout(size_t n_codes, uint64_t chunks, int64_t n_traj, int64_t shots,
                     int64_t n_kraus_pts, int kraus_gx, size_t real_bytes) {
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t T = (size_t)n_traj;
  AuxLayout a;
  a.codes = 0;
  a.seeds = up(n_codes);
  a.sums = up(a.seeds + 2 * sizeof(uint64_t));
  a.prefix = up(a.sums + sizeof(double) * chunks * T);
  a.start = up(a.prefix + sizeof(double) * chunks * T);
  a.tf = up(a.start + sizeof(double) * chunks * T);
  a.scalars = up(a.tf + sizeof(ChunkTf) * chunks * T);
  a.out = up(a.scalars + sizeof(SampleScalars) * T);
  a.partial = up(a.out + sizeof(int32_t) * (size_t)std::max<int64_t>(1, shots * n_traj));
  a.mats = up(a.partial + sizeof(double) * SC_MAX_KRAUS * (size_t)kraus_gx * T);
  a.kchoice = up(a.mats + 8 * real_bytes * T * (size_t)std::max<int64_t>(1, n_kraus_pts));
  a.status = up(a.kchoice + sizeof(int32_t) * T * (size_t)std::max<int64_t>(1, n_kraus_pts));
  a.bytes = up(a.status + sizeof(int32_t) * T);
  return a;
}

}  // namespace

// The last batch a context ran: the key it was built for, its segments (planned with
// the tile shape in force), and the CUDA graph of its device work when one was
// captured.  A call with the same circuit, records, batch size and shots reuses
// them: only the Pauli choice table and the two seeds change, and both are read from
// device memory by the graph's kernels.
struct TrajCache {
  std::vector<uint8_t> key;
  std::vector<Segment> segs;
  int tile_qubits = 0, nr = 0;  // the shape the segments were planned with
  bool tuned = false;           // shape chosen by timing the candidates
  double tuned_ms = 0.0;
  cudaGraphExec_t exec = nullptr;
  bool no_graph = false;        // capture failed once: eager launches
  void* states_p = nullptr;     // buffers the graph was captured on
  void* aux_p = nullptr;
  void* err_p = nullptr;
  int64_t launches[KC_COUNT] = {};  // kernel launches of one replay, per class

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
};

void traj_cache_free(void* p) {
  TrajCache* tc = static_cast<TrajCache*>(p);
  if (!tc) return;
  tc->drop_graph();
  delete tc;
}

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

  // Pauli decomposition of every record; the others are Kraus points
  std::vector<double> weight((size_t)n_channels * SC_MAX_KRAUS, 0.0);
  std::vector<uint8_t> code((size_t)n_channels * SC_MAX_KRAUS, 0);
  std::vector<char> is_pauli((size_t)n_channels, 1);
  std::vector<int64_t> kraus_pts;  // record index of each Kraus point, in order
  for (int64_t j = 0; j < n_channels; ++j) {
    double total = 0.0;
    for (int k = 0; k < ch[j].n_kraus && is_pauli[j]; ++k) {
      double w = 0.0;
      const int pc = pauli_of(ch[j].kraus[k], &w);
      if (pc < 0) {
        is_pauli[j] = 0;
        break;
      }
      weight[j * SC_MAX_KRAUS + k] = w;
      code[j * SC_MAX_KRAUS + k] = (uint8_t)pc;
      total += w;
    }
    if (!is_pauli[j]) {
      kraus_pts.push_back(j);
      continue;
    }
    if (!std::isfinite(total) || total <= kMinKrausWeight)
      return fail(SC_ESTATE, "noise record %lld: invalid Kraus branch weights", (long long)j);
  }
  const int64_t n_kp = (int64_t)kraus_pts.size();

  // the batch's key: everything the plans and the graph depend on except the seeds
  std::vector<uint8_t> key;
  auto put = [&](const void* d, size_t b) {
    const uint8_t* q = static_cast<const uint8_t*>(d);
    key.insert(key.end(), q, q + b);
  };
  const int64_t hdr[6] = {n, n_ops, n_channels, n_traj, shots, c->cfg.dtype};
  put(hdr, sizeof hdr);
  const int32_t knobs[6] = {c->cfg.tile_qubits, c->cfg.sweep_budget, c->low_qubits, c->nr,
                            c->rotation ? 1 : 0, c->peephole ? 1 : 0};
  put(knobs, sizeof knobs);
  put(ops, sizeof(sc_op) * (size_t)n_ops);
  put(ch.data(), sizeof(sc_channel) * ch.size());
  if (!c->traj_cache) c->traj_cache = new TrajCache();
  TrajCache* tc = static_cast<TrajCache*>(c->traj_cache);
  if (tc->key != key) {
    tc->drop_graph();
    *tc = TrajCache();
    tc->key = key;
  }

  // One gate list per segment: ops with a Pauli slot after each Pauli record.  A
  // Kraus point ends the segment; its drawn matrix is applied by a matrix record at
  // the head of the next gate list.  Back-to-back Kraus points on two qubits (the
  // records after a two-qubit gate) share one segment boundary: the second is weighed
  // with the first's matrix applied on the fly.
  auto build_segments = [&](const PlanParams& pp, std::vector<Segment>* out) -> int {
    out->clear();
    std::vector<PGate> gates;
    std::vector<std::pair<int64_t, int>> pending;  // (Kraus point, qubit) not in a list yet
    int64_t next = 0, kp_count = 0;
    auto flush_pending = [&](int64_t op) {
      for (const auto& pe : pending) {
        PGate tm;
        std::memset(&tm, 0, sizeof tm);
        tm.kind = PK_TMAT;
        tm.q0 = pe.second;
        tm.q1 = (int32_t)pe.first;
        tm.op_index = op;
        gates.push_back(tm);
      }
      pending.clear();
    };
    auto close_segment = [&](int64_t kraus, int64_t kp) -> int {
      Segment sg;
      if (!gates.empty()) {
        sg.plan = plan_sweeps(gates, n, pp);
        if (!sg.plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
      }
      sg.kraus = kraus;
      sg.kp = kp;
      if (kraus >= 0 && !pending.empty()) {
        sg.pend_kp = pending[0].first;
        sg.pend_q = pending[0].second;
      }
      out->push_back(std::move(sg));
      gates.clear();
      return SC_OK;
    };
    for (int64_t i = 0; i < n_ops; ++i) {
      PGate g;
      bool produced = false;
      if (!normalise_op(ops[i], nullptr, 0, &g, &produced))
        return fail(SC_EINVAL, "op %lld: cannot normalise", (long long)i);
      if (produced) {
        flush_pending(i);
        g.op_index = i;
        gates.push_back(g);
      }
      while (next < n_channels && ch[next].after_op == i) {
        if (is_pauli[next]) {
          flush_pending(i);
          PGate sl;
          std::memset(&sl, 0, sizeof sl);
          sl.kind = PK_PAULI;
          sl.q0 = ch[next].target;
          sl.q1 = (int32_t)next;
          sl.op_index = i;
          gates.push_back(sl);
        } else {
          const int q = ch[next].target;
          if (pending.size() > 1 || (pending.size() == 1 && pending[0].second == q))
            flush_pending(i);
          const int r = close_segment(next, kp_count);
          if (r != SC_OK) return r;
          pending.emplace_back(kp_count++, q);
        }
        ++next;
      }
    }
    flush_pending(n_ops - 1);
    if (!gates.empty()) return close_segment(-1, -1);
    return SC_OK;
  };
  auto shape_params = [&](int tile, int nr) {
    PlanParams pp = c->plan_params();
    pp.relayout = false;  // each segment is planned alone; no layout to restore
    if (tile > 0) pp.tile_qubits = tile;
    if (nr > 0) pp.nr = nr;
    return pp;
  };

  // branch choices of the Pauli records, drawn as the reference draws them
  const size_t n_ch = (size_t)n_channels;
  std::vector<uint8_t> paulis(std::max<size_t>(1, (size_t)n_traj * n_ch), 0);
  for (int64_t t = 0; t < n_traj; ++t) {
    const uint64_t seed = noise_seed + (uint64_t)t;
    for (size_t j = 0; j < n_ch; ++j) {
      if (!is_pauli[j]) continue;
      const double* w = &weight[j * SC_MAX_KRAUS];
      double total = 0.0;
      for (int k = 0; k < ch[j].n_kraus; ++k) total += w[k];
      const int idx = weighted_index(w, ch[j].n_kraus, next_double_bound(seed, j, total));
      paulis[(size_t)t * n_ch + j] = code[j * SC_MAX_KRAUS + idx];
      if (choices) choices[(size_t)t * n_ch + j] = idx;
    }
  }

  // device buffers: states; codes | seeds | sampling scratch | outcomes | Kraus scratch
  const size_t amp = c->cfg.dtype == SC_C64 ? 8 : 16;
  const uint64_t len = 1ULL << n;
  const size_t state_bytes = amp * len * (size_t)n_traj;
  const uint64_t chunks = sample_chunks(len);
  const int kraus_gx = noise_grid_batch(n, n_traj, c->sm_count);
  const AuxLayout L = aux_layout(paulis.size(), chunks, n_traj, shots, n_kp, kraus_gx, amp / 2);
  if ((rc = c->reserve(c->buf_traj_states, state_bytes, "trajectory states")) != SC_OK) return rc;
  if ((rc = c->reserve(c->buf_traj_aux, L.bytes, "trajectory scratch")) != SC_OK) return rc;
  if ((rc = c->reserve(c->buf_err, 16, "error flag")) != SC_OK) return rc;
  char* aux = static_cast<char*>(c->buf_traj_aux.p);
  cudaStream_t s = c->stream;
  const uint64_t seeds[2] = {noise_seed, measure_seed};
  cudaError_t e = cudaMemcpyAsync(aux + L.codes, paulis.data(), paulis.size(),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(aux + L.seeds, seeds, sizeof seeds, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail_cuda(e, "trajectory set-up");

  const double dim = std::ldexp(1.0, n);
  const uint64_t* seeds_dev = reinterpret_cast<const uint64_t*>(aux + L.seeds);
  int32_t* status_dev = reinterpret_cast<int32_t*>(aux + L.status);
  SampleArgs sa;
  sa.chunk_sums = reinterpret_cast<double*>(aux + L.sums);
  sa.chunk_prefix = reinterpret_cast<double*>(aux + L.prefix);
  sa.chunk_start = reinterpret_cast<double*>(aux + L.start);
  sa.chunk_tf = reinterpret_cast<ChunkTf*>(aux + L.tf);
  sa.scalars = reinterpret_cast<SampleScalars*>(aux + L.scalars);
  sa.uniforms = nullptr;
  sa.seed = measure_seed;
  sa.seed_dev = seeds_dev + 1;
  sa.shots = shots;
  sa.outcomes = reinterpret_cast<int32_t*>(aux + L.out);
  sa.sm_count = c->sm_count;

  // the device work of one batch: |0..0> in every state, each segment's sweeps and
  // Kraus point, then the sampling of every state
  auto enqueue = [&](const std::vector<Segment>& segs, bool sample) -> cudaError_t {
    cudaError_t r = cudaMemsetAsync(c->buf_err.p, 0, 16, s);
    if (r == cudaSuccess) r = cudaMemsetAsync(status_dev, 0, sizeof(int32_t) * (size_t)n_traj, s);
    if (r != cudaSuccess) return r;
    c->mark_begin(KC_INIT, dim * (double)amp * (double)n_traj);
    r = launch_init_batch(c->cfg.dtype, c->buf_traj_states.p, n, n_traj, s);
    c->mark_end();
    if (r != cudaSuccess) return r;
    for (const Segment& sg : segs) {
      for (size_t k = 0; k < sg.plan.sweeps.size(); ++k) {
        c->mark_begin(KC_SWEEP, 2.0 * dim * (double)amp * (double)n_traj);
        r = launch_sweep_batch(c->cfg.dtype, c->buf_traj_states.p, n, n_traj, sg.plan, k,
                               reinterpret_cast<const uint8_t*>(aux + L.codes), (int)n_ch,
                               aux + L.mats, static_cast<int*>(c->buf_err.p), c->sm_count, s);
        c->mark_end();
        if (r != cudaSuccess) return r;
      }
      if (sg.kraus < 0) continue;
      const sc_channel& rec = ch[(size_t)sg.kraus];
      KrausArgs ka;
      std::memset(&ka, 0, sizeof ka);
      ka.nk = rec.n_kraus;
      ka.target = rec.target;
      for (int k = 0; k < rec.n_kraus; ++k) std::memcpy(ka.k[k], rec.kraus[k], 8 * sizeof(double));
      const size_t mat_bytes = 4 * amp * (size_t)n_traj;  // one Kraus point's matrices
      c->mark_begin(KC_NOISE, dim * (double)amp * (double)n_traj, 2);
      r = launch_kraus_batch(c->cfg.dtype, c->buf_traj_states.p, n, n_traj, ka, sg.pend_q,
                             sg.pend_kp >= 0 ? aux + L.mats + sg.pend_kp * mat_bytes : nullptr,
                             seeds_dev, (uint64_t)sg.kraus,
                             reinterpret_cast<double*>(aux + L.partial),
                             aux + L.mats + sg.kp * mat_bytes,
                             reinterpret_cast<int32_t*>(aux + L.kchoice) + sg.kp, n_kp, status_dev,
                             c->sm_count, s);
      c->mark_end();
      if (r != cudaSuccess) return r;
    }
    if (sample && shots > 0) {
      c->mark_begin(KC_SAMPLE, dim * (double)amp * (double)n_traj, kSampleKernels);
      r = launch_sample_batch(c->cfg.dtype, c->buf_traj_states.p, len, n_traj, sa, s);
      c->mark_end();
    }
    return r;
  };

  // the tile shape: the context's, or (autotune) the fastest of a few candidates,
  // timed on this batch once per key
  if (tc->segs.empty()) {
    const PlanParams base = c->plan_params();
    int best_tile = base.tile_qubits, best_nr = base.nr;
    if (c->cfg.autotune && !tc->tuned) {
      const int cand[4][2] = {{base.tile_qubits, base.nr}, {base.tile_qubits + 1, base.nr},
                              {base.tile_qubits - 1, base.nr}, {base.tile_qubits, 3}};
      float best_ms = 0.0f;
      cudaEvent_t e0 = c->get_event(), e1 = c->get_event();
      // the tuning runs stay out of the launch counts and per-class times
      int64_t saved[KC_COUNT];
      std::memcpy(saved, c->stats_launch, sizeof saved);
      const int timing = c->cfg.timing;
      c->cfg.timing = 0;
      for (const auto& cd : cand) {
        if (cd[0] > n || cd[0] < 6 || cd[1] < 2 || cd[1] > 4) continue;
        std::vector<Segment> segs;
        if (build_segments(shape_params(cd[0], cd[1]), &segs) != SC_OK) continue;
        float ms = -1.0f;
        for (int rep = 0; rep < 2; ++rep) {  // the first run loads the kernels
          if (cudaEventRecord(e0, s) != cudaSuccess) break;
          if (enqueue(segs, false) != cudaSuccess) {
            ms = -1.0f;
            break;
          }
          cudaEventRecord(e1, s);
          if (cudaEventSynchronize(e1) != cudaSuccess) break;
          cudaEventElapsedTime(&ms, e0, e1);
        }
        cudaGetLastError();  // a shape the kernels reject is skipped
        if (ms > 0.0f && (best_ms == 0.0f || ms < best_ms)) {
          best_ms = ms;
          best_tile = cd[0];
          best_nr = cd[1];
        }
      }
      c->cfg.timing = timing;
      std::memcpy(c->stats_launch, saved, sizeof saved);
      tc->tuned = true;
      tc->tuned_ms = best_ms;
    }
    if ((rc = build_segments(shape_params(best_tile, best_nr), &tc->segs)) != SC_OK) return rc;
    tc->tile_qubits = best_tile;
    tc->nr = best_nr;
  }

  // the graph: captured once per key and buffer set (not while timing per kernel)
  bool use_graph = !c->cfg.timing && !tc->no_graph;
  if (use_graph && tc->exec &&
      (tc->states_p != c->buf_traj_states.p || tc->aux_p != c->buf_traj_aux.p ||
       tc->err_p != c->buf_err.p))
    tc->drop_graph();
  if (use_graph && !tc->exec) {
    int64_t before[KC_COUNT];
    std::memcpy(before, c->stats_launch, sizeof before);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      const cudaError_t qe = enqueue(tc->segs, true);
      ce = cudaStreamEndCapture(s, &g);
      if (ce == cudaSuccess) ce = qe;
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&tc->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    for (int k = 0; k < KC_COUNT; ++k) {
      tc->launches[k] = c->stats_launch[k] - before[k];
      c->stats_launch[k] = before[k];
    }
    if (ce != cudaSuccess) {
      cudaGetLastError();
      tc->exec = nullptr;
      tc->no_graph = true;
      use_graph = false;
    } else {
      tc->states_p = c->buf_traj_states.p;
      tc->aux_p = c->buf_traj_aux.p;
      tc->err_p = c->buf_err.p;
    }
  }
  if (use_graph) {
    e = cudaGraphLaunch(tc->exec, s);
    if (e == cudaSuccess)
      for (int k = 0; k < KC_COUNT; ++k) c->stats_launch[k] += tc->launches[k];
  } else {
    e = enqueue(tc->segs, true);
  }
  if (e != cudaSuccess) return fail_cuda(e, "trajectory batch");

  std::vector<SampleScalars> scal((size_t)n_traj);
  std::vector<int32_t> status((size_t)n_traj, 0);
  std::vector<int32_t> kchoice((size_t)n_traj * (size_t)std::max<int64_t>(1, n_kp), 0);
  e = cudaMemcpyAsync(status.data(), status_dev, sizeof(int32_t) * status.size(),
                      cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && n_kp > 0)
    e = cudaMemcpyAsync(kchoice.data(), aux + L.kchoice, sizeof(int32_t) * kchoice.size(),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && shots > 0)
    e = cudaMemcpyAsync(scal.data(), sa.scalars, sizeof(SampleScalars) * scal.size(),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && shots > 0)
    e = cudaMemcpyAsync(outcomes, sa.outcomes, sizeof(int32_t) * (size_t)(shots * n_traj),
                        cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return fail_cuda(e, "outcome download");
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
  for (int64_t t = 0; t < n_traj; ++t) {
    if (status[t] == kNoiseBadWeight || status[t] == kNoiseBadTotal)
      return fail(SC_ESTATE, "trajectory %lld: invalid Kraus branch weights", (long long)t);
    if (status[t] != 0)
      return fail(SC_ESTATE, "trajectory %lld: state norm is zero after a Kraus operator",
                  (long long)t);
  }
  for (int64_t t = 0; t < (shots > 0 ? n_traj : 0); ++t)
    if (scal[t].status != 0)
      return fail(SC_ESTATE, "trajectory %lld: state collapsed to zero probability amplitudes",
                  (long long)t);
  if (choices)
    for (int64_t t = 0; t < n_traj; ++t)
      for (int64_t q = 0; q < n_kp; ++q)
        choices[(size_t)t * n_ch + (size_t)kraus_pts[q]] = kchoice[(size_t)t * n_kp + q];
  c->plan_sweeps_count = c->plan_gates = c->plan_stages = 0;
  for (const Segment& sg : tc->segs) {
    c->plan_sweeps_count += (int64_t)sg.plan.sweeps.size();
    c->plan_gates += sg.plan.n_gates;
    c->plan_stages += (int64_t)sg.plan.stages.size();
  }
  return SC_OK;
}

int32_t sc_trajectories_info(void* p, int32_t* tile_qubits, int32_t* nr, int32_t* graph,
                             double* tuned_ms) {
  int rc = check_context(p);
  if (rc != SC_OK) return rc;
  const TrajCache* tc = static_cast<const TrajCache*>(static_cast<Ctx*>(p)->traj_cache);
  if (tile_qubits) *tile_qubits = tc ? tc->tile_qubits : 0;
  if (nr) *nr = tc ? tc->nr : 0;
  if (graph) *graph = (tc && tc->exec) ? 1 : 0;
  if (tuned_ms) *tuned_ms = tc ? tc->tuned_ms : 0.0;
  return SC_OK;
}

}  // extern "C"
