// Batched QAOA ring ansatz (host side): instance layout in HBM, phase / RX
// tables, the pass schedule, a small autotuner over kernel shapes, and the CUDA
// graph that replays one whole batch with a single launch.
//
// The reference runs such a suite one circuit at a time through
// StatevectorEngine.simulate (app/.../AlgorithmSuiteSpecs.java:186-200 builds the
// ansatz); this batch object has no reference counterpart.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sc_ctx.h"
#include "sc_qaoa.h"

namespace sc {

struct QaoaBatch {
  static constexpr uint32_t kMagic = 0x9a0a7b01u;
  uint32_t magic = kMagic;
  Ctx* ctx = nullptr;
  int dtype = SC_C128;
  int p = 0;
  int64_t n_inst = 0;
  std::vector<int32_t> nq;
  std::vector<QaoaInst> large, whole;
  std::vector<int64_t> lprefix, wprefix;
  std::vector<QaoaSpan> spans;
  int64_t n_items_large = 0;
  int64_t arena_amps = 0;
  int64_t n_phase = 0;  // complex entries
  DevBuf d_state, d_large, d_whole, d_lprefix, d_wprefix, d_cs, d_escale, d_phase, d_partials,
      d_spans, d_energy, d_norm;
  int shape = 1;
  int ctas = 1;
  double tuned_ms = 0.0;
  double bytes_per_run = 0.0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;

  void free_all() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    for (DevBuf* b : {&d_state, &d_large, &d_whole, &d_lprefix, &d_wprefix, &d_cs, &d_escale,
                      &d_phase, &d_partials, &d_spans, &d_energy, &d_norm})
      ctx->release(*b);
  }
};

void qaoa_batch_free(void* b) {
  QaoaBatch* q = static_cast<QaoaBatch*>(b);
  if (!q) return;
  q->free_all();
  q->magic = 0;
  delete q;
}

namespace {

QaoaBatch* as_batch(void* p) {
  QaoaBatch* q = static_cast<QaoaBatch*>(p);
  if (!q || q->magic != QaoaBatch::kMagic) return nullptr;
  if (cudaSetDevice(q->ctx->device) != cudaSuccess) return nullptr;
  return q;
}

int upload(Ctx* c, DevBuf& b, const void* src, size_t bytes, const char* what) {
  int rc = c->reserve(b, std::max<size_t>(bytes, 16), what);
  if (rc != SC_OK) return rc;
  if (bytes == 0) return SC_OK;
  cudaError_t e = cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream);
  return e == cudaSuccess ? SC_OK : fail_cuda(e, what);
}

// RX coefficients and cost-phase tables from the angles, in FP64 on the host.
//
// RX(2b) = c I - i s X (c = cos b, s = sin b) is applied as a scalar times a
// matrix with one unit diagonal or off-diagonal: c (I - i t X), t = s / c, when
// |c| >= |s|, else s (u I - i X), u = c / s.  A layer half acting on k qubits then
// leaves the scalar sc^k, which is folded into the next cost-phase table (a
// pass applies RX of layer l-1 on its half, the phase of layer l, RX of layer l
// on its half) or, after the last layer, into the energy (squared).
int fill_angles(QaoaBatch* q, const double* gammas, const double* betas) {
  const int p = q->p;
  std::vector<double> cs(2 * (size_t)q->n_inst * p);
  std::vector<double> scal((size_t)q->n_inst * p);
  std::vector<double> ph(2 * (size_t)q->n_phase);
  std::vector<double> escale((size_t)q->n_inst, 1.0);
  for (int64_t i = 0; i < q->n_inst; ++i)
    for (int l = 0; l < p; ++l) {
      const double b = betas[(size_t)i * p + l];
      const double c = std::cos(b), s = std::sin(b);
      const size_t at = (size_t)i * p + l;
      if (std::fabs(c) >= std::fabs(s)) {
        cs[2 * at] = s / c;
        cs[2 * at + 1] = 0.0;
        scal[at] = c;
      } else {
        cs[2 * at] = c / s;
        cs[2 * at + 1] = 1.0;
        scal[at] = s;
      }
    }
  // half_bits(k): qubits the RX layers of pass k act on; whole instances apply
  // every layer to all n qubits in one go
  auto put_tables = [&](const QaoaInst& in, bool whole) {
    const size_t base = (size_t)in.orig * p;
    auto half_bits = [&](int k) {
      if (whole) return in.n;
      return (k & 1) ? in.n - kQaoaTileQubits : kQaoaTileQubits;
    };
    for (int l = 0; l < p; ++l) {
      const double g = gammas[base + l];
      // scalars folded into this table: RX of layer l-1 and (pass form) layer l
      double f = 1.0;
      if (whole) {
        if (l > 0) f = std::pow(scal[base + l - 1], in.n);
      } else {
        const int bits = half_bits(l);
        f = std::pow(scal[base + l], bits);
        if (l > 0) f *= std::pow(scal[base + l - 1], bits);
      }
      for (int k = 0; k <= in.n; ++k) {
        // exp(-i gamma sum_j z_j z_{j+1}) with sum = n - 2k
        const double a = -g * (double)(in.n - 2 * k);
        const size_t at = 2 * (size_t)(in.ph_off + (int64_t)l * (in.n + 1) + k);
        ph[at] = f * std::cos(a);
        ph[at + 1] = f * std::sin(a);
      }
    }
    const double last = std::pow(scal[base + p - 1], whole ? in.n : half_bits(p));
    escale[in.orig] = last * last;
  };
  for (const QaoaInst& in : q->large) put_tables(in, false);
  for (const QaoaInst& in : q->whole) put_tables(in, true);
  int rc = upload(q->ctx, q->d_cs, cs.data(), cs.size() * sizeof(double), "QAOA RX table");
  if (rc == SC_OK)
    rc = upload(q->ctx, q->d_escale, escale.data(), escale.size() * sizeof(double), "QAOA scales");
  if (rc != SC_OK) return rc;
  return upload(q->ctx, q->d_phase, ph.data(), ph.size() * sizeof(double), "QAOA phase table");
}

int enqueue(QaoaBatch* q, int shape, int ctas) {
  Ctx* c = q->ctx;
  cudaError_t e;
  QaoaLaunch a;
  std::memset(&a, 0, sizeof a);
  a.state = q->d_state.p;
  a.p = q->p;
  a.cs = static_cast<const double*>(q->d_cs.p);
  a.escale = static_cast<const double*>(q->d_escale.p);
  a.phase = static_cast<const double*>(q->d_phase.p);
  a.partials = static_cast<double*>(q->d_partials.p);
  if (!q->whole.empty()) {
    QaoaLaunch w = a;
    w.inst = static_cast<const QaoaInst*>(q->d_whole.p);
    w.item_prefix = static_cast<const int64_t*>(q->d_wprefix.p);
    w.n_inst = (int32_t)q->whole.size();
    w.n_items = (int64_t)q->whole.size();
    w.part_base = q->n_items_large;
    QaoaPass pw{kQaoaWhole, 1, -1, -1, -1, 1};
    if ((e = launch_qaoa(q->dtype, shape, w, pw, ctas, c->sm_count, c->stream)) != cudaSuccess)
      return fail_cuda(e, "QAOA whole-instance kernel");
  }
  if (!q->large.empty()) {
    QaoaLaunch l = a;
    l.inst = static_cast<const QaoaInst*>(q->d_large.p);
    l.item_prefix = static_cast<const int64_t*>(q->d_lprefix.p);
    l.n_inst = (int32_t)q->large.size();
    l.n_items = q->n_items_large;
    l.part_base = 0;
    for (int k = 0; k <= q->p; ++k) {
      QaoaPass ps;
      ps.mode = (k & 1) ? kQaoaHigh : kQaoaLow;
      ps.init = k == 0;
      ps.rx_a = k > 0 ? k - 1 : -1;
      ps.d = k < q->p ? k : -1;
      ps.rx_b = k < q->p ? k : -1;
      ps.reduce = k == q->p;
      if ((e = launch_qaoa(q->dtype, shape, l, ps, ctas, c->sm_count, c->stream)) != cudaSuccess)
        return fail_cuda(e, "QAOA pass kernel");
    }
  }
  e = launch_qaoa_reduce(static_cast<const double*>(q->d_partials.p),
                         static_cast<const QaoaSpan*>(q->d_spans.p), q->n_inst,
                         static_cast<double*>(q->d_energy.p), static_cast<double*>(q->d_norm.p),
                         c->stream);
  return e == cudaSuccess ? SC_OK : fail_cuda(e, "QAOA energy reduction");
}

// Times every kernel shape (register group width and register budget) at every
// launchable number of resident CTAs per SM on the batch itself; keeps the fastest.
int autotune(QaoaBatch* q) {
  Ctx* c = q->ctx;
  cudaEvent_t e0 = c->get_event(), e1 = c->get_event();
  double best = 1e300;
  int best_shape = 1, best_ctas = 1;
  for (int shape = 0; shape < kQaoaShapes; ++shape) {
    const int most = qaoa_max_ctas_per_sm(q->dtype, shape, q->p);
    for (int ctas = 1; ctas <= most; ++ctas) {
      int rc = enqueue(q, shape, ctas);  // warm-up
      if (rc != SC_OK) return rc;
      cudaEventRecord(e0, c->stream);
      for (int r = 0; r < 2; ++r)
        if ((rc = enqueue(q, shape, ctas)) != SC_OK) return rc;
      cudaEventRecord(e1, c->stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return fail_cuda(e, "QAOA autotune");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms / 2.0 < best) {
        best = ms / 2.0;
        best_shape = shape;
        best_ctas = ctas;
      }
    }
  }
  q->shape = best_shape;
  q->ctas = best_ctas;
  q->tuned_ms = best;
  return SC_OK;
}

int capture(QaoaBatch* q) {
  Ctx* c = q->ctx;
  // function attributes are set outside the capture
  if (qaoa_max_ctas_per_sm(q->dtype, q->shape, q->p) <= 0)
    return fail(SC_ECUDA, "QAOA kernel shape not launchable");
  cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail_cuda(e, "QAOA graph capture");
  int rc = enqueue(q, q->shape, q->ctas);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(c->stream, &g);
  if (rc != SC_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail_cuda(e, "QAOA graph capture");
  q->graph = g;
  e = cudaGraphInstantiate(&q->exec, g, 0);
  if (e != cudaSuccess) return fail_cuda(e, "QAOA graph instantiate");
  return SC_OK;
}

}  // namespace
}  // namespace sc

using namespace sc;

extern "C" {

int32_t sc_qaoa_batch_create(void* ctx, int32_t dtype, int64_t n_inst, const int32_t* n_qubits,
                             int32_t p, const double* gammas, const double* betas, int32_t tune,
                             void** out_batch) {
  Ctx* c = static_cast<Ctx*>(ctx);
  if (!c || c->magic != Ctx::kMagic) return fail(SC_EINVAL, "invalid context");
  if (!out_batch) return fail(SC_EINVAL, "out_batch is null");
  {
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  }
  *out_batch = nullptr;
  if (dtype != SC_C128 && dtype != SC_C64) return fail(SC_EINVAL, "unknown dtype %d", dtype);
  if (n_inst < 1 || !n_qubits || !gammas || !betas)
    return fail(SC_EINVAL, "empty batch or null input");
  if (p < 1 || p > kQaoaMaxLayers)
    return fail(SC_EINVAL, "layer count %d outside 1..%d", p, kQaoaMaxLayers);
  if (n_inst > (1LL << 30)) return fail(SC_EINVAL, "too many instances");
  for (int64_t i = 0; i < n_inst; ++i)
    if (n_qubits[i] < 2 || n_qubits[i] > kQaoaMaxQubits)
      return fail(SC_EINVAL, "instance %lld: %d qubits outside 2..%d", (long long)i, n_qubits[i],
                  kQaoaMaxQubits);
  QaoaBatch* q = new QaoaBatch();
  q->ctx = c;
  q->dtype = dtype;
  q->p = p;
  q->n_inst = n_inst;
  q->nq.assign(n_qubits, n_qubits + n_inst);

  // large instances first, largest first (the long tiles of a launch start early)
  std::vector<int64_t> order(n_inst);
  for (int64_t i = 0; i < n_inst; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t a, int64_t b) { return n_qubits[a] > n_qubits[b]; });
  const size_t amp_bytes = dtype == SC_C64 ? 8 : 16;
  int64_t ph_off = 0;
  q->spans.assign(n_inst, QaoaSpan{0, 0});
  q->lprefix.push_back(0);
  q->wprefix.push_back(0);
  for (int64_t oi : order) {
    QaoaInst in;
    in.n = n_qubits[oi];
    in.orig = (int32_t)oi;
    in.ph_off = ph_off;
    ph_off += (int64_t)p * (in.n + 1);
    if (in.n > kQaoaTileQubits) {
      in.amp_off = q->arena_amps;
      q->arena_amps += 1LL << in.n;
      const int64_t items = 1LL << (in.n - kQaoaTileQubits);
      q->spans[oi] = QaoaSpan{q->n_items_large, q->n_items_large + items};
      q->n_items_large += items;
      q->lprefix.push_back(q->n_items_large);
      q->large.push_back(in);
      q->bytes_per_run += 2.0 * p * (double)amp_bytes * std::ldexp(1.0, in.n);
    } else {
      in.amp_off = 0;
      q->whole.push_back(in);
      q->wprefix.push_back((int64_t)q->whole.size());
    }
  }
  for (int64_t k = 0; k < (int64_t)q->whole.size(); ++k) {
    const int32_t oi = q->whole[k].orig;
    q->spans[oi] = QaoaSpan{q->n_items_large + k, q->n_items_large + k + 1};
  }
  q->n_phase = ph_off;

  int rc = c->reserve(q->d_state, std::max<size_t>(16, amp_bytes * (size_t)q->arena_amps),
                      "QAOA batch states");
  if (rc == SC_OK) rc = upload(c, q->d_large, q->large.data(), q->large.size() * sizeof(QaoaInst), "QAOA instances");
  if (rc == SC_OK) rc = upload(c, q->d_whole, q->whole.data(), q->whole.size() * sizeof(QaoaInst), "QAOA instances");
  if (rc == SC_OK) rc = upload(c, q->d_lprefix, q->lprefix.data(), q->lprefix.size() * sizeof(int64_t), "QAOA items");
  if (rc == SC_OK) rc = upload(c, q->d_wprefix, q->wprefix.data(), q->wprefix.size() * sizeof(int64_t), "QAOA items");
  if (rc == SC_OK) rc = upload(c, q->d_spans, q->spans.data(), q->spans.size() * sizeof(QaoaSpan), "QAOA spans");
  if (rc == SC_OK)
    rc = c->reserve(q->d_partials, 2 * sizeof(double) * (size_t)(q->n_items_large + q->whole.size()),
                    "QAOA partial sums");
  if (rc == SC_OK) rc = c->reserve(q->d_energy, sizeof(double) * (size_t)n_inst, "QAOA energies");
  if (rc == SC_OK) rc = c->reserve(q->d_norm, sizeof(double) * (size_t)n_inst, "QAOA norms");
  if (rc == SC_OK) rc = fill_angles(q, gammas, betas);
  if (rc == SC_OK) {
    if (tune) {
      rc = autotune(q);
    } else {
      q->shape = 0;
      q->ctas = std::max(1, qaoa_max_ctas_per_sm(dtype, 0, p));
    }
  }
  if (rc == SC_OK) rc = capture(q);
  if (rc == SC_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) rc = fail_cuda(e, "QAOA batch set-up");
  }
  if (rc != SC_OK) {
    qaoa_batch_free(q);
    return rc;
  }
  c->qaoa_batches.push_back(q);
  *out_batch = q;
  return SC_OK;
}

int32_t sc_qaoa_batch_set_angles(void* batch, const double* gammas, const double* betas) {
  QaoaBatch* q = as_batch(batch);
  if (!q) return fail(SC_EINVAL, "invalid QAOA batch");
  if (!gammas || !betas) return fail(SC_EINVAL, "null angles");
  return fill_angles(q, gammas, betas);
}

int32_t sc_qaoa_batch_run(void* batch) {
  QaoaBatch* q = as_batch(batch);
  if (!q) return fail(SC_EINVAL, "invalid QAOA batch");
  Ctx* c = q->ctx;
  c->mark_begin(KC_BATCH, q->bytes_per_run,
                (int)(q->large.empty() ? 0 : q->p + 1) + (q->whole.empty() ? 0 : 1) + 1);
  cudaError_t e = cudaGraphLaunch(q->exec, c->stream);
  c->mark_end();
  return e == cudaSuccess ? SC_OK : fail_cuda(e, "QAOA graph launch");
}

int32_t sc_qaoa_batch_energies(void* batch, double* energies, double* norms) {
  QaoaBatch* q = as_batch(batch);
  if (!q) return fail(SC_EINVAL, "invalid QAOA batch");
  Ctx* c = q->ctx;
  cudaError_t e = cudaSuccess;
  if (energies)
    e = cudaMemcpyAsync(energies, q->d_energy.p, sizeof(double) * (size_t)q->n_inst,
                        cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && norms)
    e = cudaMemcpyAsync(norms, q->d_norm.p, sizeof(double) * (size_t)q->n_inst,
                        cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail_cuda(e, "QAOA energies");
  c->collect_timing();
  return SC_OK;
}

int32_t sc_qaoa_batch_info(void* batch, int32_t* nr, int32_t* ctas_per_sm, double* tuned_ms,
                           double* bytes_per_run) {
  QaoaBatch* q = as_batch(batch);
  if (!q) return fail(SC_EINVAL, "invalid QAOA batch");
  if (nr) *nr = qaoa_shape_nr(q->shape);
  if (ctas_per_sm) *ctas_per_sm = q->ctas;
  if (tuned_ms) *tuned_ms = q->tuned_ms;
  if (bytes_per_run) *bytes_per_run = q->bytes_per_run;
  return SC_OK;
}

int32_t sc_qaoa_batch_destroy(void* batch) {
  QaoaBatch* q = as_batch(batch);
  if (!q) return batch ? fail(SC_EINVAL, "invalid QAOA batch") : SC_OK;
  Ctx* c = q->ctx;
  cudaStreamSynchronize(c->stream);
  auto& v = c->qaoa_batches;
  v.erase(std::remove(v.begin(), v.end(), static_cast<void*>(q)), v.end());
  qaoa_batch_free(q);
  return SC_OK;
}

}  // extern "C"
