// Adjoint differentiation entry points (addition; the reference engine has no
// gradient API).  Two device state buffers (psi, lambda), no stored intermediate
// states: the reverse pass un-applies each gate from both.  When the circuit fits
// (1-qubit rotation generators, no dense 2-qubit gates) the reverse pass runs as
// fused dual-state sweeps, each carrying both states through many inverse gates
// and gradient probes; otherwise gate by gate, three passes per rotation.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sc_adjoint.h"
#include "sc_ctx.h"
#include "sc_sweep.h"

namespace sc {

namespace {

void conj_transpose(const double* m, int dim, double* out) {
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) {
      out[2 * (dim * c + r)] = m[2 * (dim * r + c)];
      out[2 * (dim * c + r) + 1] = -m[2 * (dim * r + c) + 1];
    }
}

PGate invert(const PGate& g) {
  PGate h = g;
  switch (g.kind) {
    case PK_DENSE1: conj_transpose(g.m, 2, h.m); break;
    case PK_DENSE2: conj_transpose(g.m, 4, h.m); break;
    case PK_DIAG1:
      for (int k = 1; k < 4; k += 2) h.m[k] = -g.m[k];
      break;
    case PK_DIAG2:
      for (int k = 1; k < 8; k += 2) h.m[k] = -g.m[k];
      break;
    default: break;  // X and SWAP are self-inverse
  }
  return h;
}

bool generator(const sc_op& op, uint64_t* x, uint64_t* z) {
  switch (op.kind) {
    case SC_OP_RX: *x = 1ULL << op.q0; *z = 0; return true;
    case SC_OP_RY: *x = 1ULL << op.q0; *z = 1ULL << op.q0; return true;  // Y = i X Z
    case SC_OP_RZ: *x = 0; *z = 1ULL << op.q0; return true;
    case SC_OP_RZZ: *x = 0; *z = (1ULL << op.q0) | (1ULL << op.q1); return true;
    default: return false;
  }
}

// The inverse gates in reverse order, with a probe before each parametrised gate
// (gradient slot = the op's parameter index).  Within a run of parametrised
// rotations on distinct qubits all probes come first: a probe on qubit q commutes
// with gates on other qubits (they act on both states), so the inverse rotations
// of the run stay adjacent and group into one record per stage.  False when some
// generator is not a single-qubit Pauli (the gate-by-gate path handles those).
bool reverse_gates(const Ctx* c, std::vector<PGate>& out) {
  std::vector<PGate> probes, gates;
  uint64_t run_qubits = 0;
  auto flush = [&]() {
    out.insert(out.end(), probes.begin(), probes.end());
    out.insert(out.end(), gates.begin(), gates.end());
    probes.clear();
    gates.clear();
    run_qubits = 0;
  };
  for (int64_t i = (int64_t)c->adj_ops.size() - 1; i >= 0; --i) {
    const sc_op& op = c->adj_ops[i];
    if (op.kind == SC_OP_MEASURE) continue;
    PGate g;
    bool produced = false;
    normalise_op(op, c->adj_params.data(), (int64_t)c->adj_params.size(), &g, &produced);
    if (!produced) continue;
    PGate inv = invert(g);
    inv.op_index = i;
    uint64_t x = 0, z = 0;
    if (op.param >= 0 && generator(op, &x, &z)) {
      const uint64_t q = x | z;
      if (__builtin_popcountll(q) != 1) return false;
      if (run_qubits & q || (touch_mask(inv) & ~q)) flush();
      PGate pr;
      std::memset(&pr, 0, sizeof pr);
      pr.kind = PK_PROBE;
      pr.q0 = __builtin_ctzll(q);
      pr.q1 = x ? (z ? 2 : 1) : 3;  // X, Y = iXZ, Z
      pr.op_index = op.param;
      probes.push_back(pr);
      gates.push_back(inv);
      run_qubits |= q;
      continue;
    }
    flush();
    out.push_back(inv);
  }
  flush();
  return true;
}

// doubles of partial sums in buf_adj_phi ahead of the gradient: per block of the
// inner-product kernels (gate-by-gate path, <H>) or per CTA and probe of a fused
// reverse sweep
size_t partial_doubles(const Ctx* c) {
  const int blocks = adjoint_partial_blocks(c->n, c->sm_count);
  return std::max<size_t>(2 * (size_t)blocks, (size_t)c->sm_count * 8 * (size_t)kSweepMaxGates);
}

int reserve_scratch(Ctx* c, int64_t n_params) {
  return c->reserve(c->buf_adj_phi, sizeof(double) * (partial_doubles(c) + (size_t)(n_params + 1)),
                    "adjoint scratch");
}

// Sweep shape of the reverse pass: 3 register qubits (both states' registers in one
// thread), phase-free records (lifted rotations, half diagonals) and plain matrix
// records; 2048-amplitude tiles (256 threads) unless
// STATECRAFT_B200_ADJOINT_TILE sets the tile qubits (10: 128-thread tiles).
PlanParams reverse_plan_params(const Ctx* c) {
  PlanParams pp;
  const bool c64 = c->cfg.dtype == SC_C64;
  pp.tile_qubits = 11;
  if (const char* v = getenv("STATECRAFT_B200_ADJOINT_TILE")) {
    const int t = atoi(v);
    if (t >= 8 && t <= 11) pp.tile_qubits = t;
  }
  pp.low_qubits = c64 ? 5 : 4;
  pp.nr = 3;
  pp.budget = -1.0;
  pp.max_gates = kSweepMaxGates;
  pp.max_pool = kSweepMaxPool;
  pp.relayout = false;
  pp.rot_min_c = 0.0;
  pp.peephole = false;
  // both states take every gate: phases common to a gate cancel in the probes, so
  // real rotations run as lifting shears and 1-qubit diagonals as diag(1, d)
  pp.phase_free = true;
  pp.entry_fold = c->entry_fold;
  return pp;
}

}  // namespace

}  // namespace sc

using namespace sc;

extern "C" {

int32_t sc_adjoint_forward(void* p, int32_t n_qubits, const sc_op* ops, int64_t n_ops,
                           const double* params, int64_t n_params, int32_t n_terms,
                           const uint64_t* xmask, const uint64_t* zmask, const double* coeffs,
                           double* out_value) {
  Ctx* c = static_cast<Ctx*>(p);
  if (!c || c->magic != Ctx::kMagic) return fail(SC_EINVAL, "invalid context handle");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(SC_ECUDA, "cudaSetDevice failed");
  c->adj_ready = false;
  if (!c->noise.empty())
    return fail(SC_EUNSUPPORTED, "adjoint differentiation requires a noiseless circuit");
  if (n_params < 0 || (n_params > 0 && !params)) return fail(SC_EINVAL, "invalid parameter vector");
  if (n_terms < 0 || (n_terms > 0 && (!xmask || !zmask || !coeffs)))
    return fail(SC_EINVAL, "invalid Hamiltonian arrays");
  for (int64_t i = 0; i < n_ops && ops; ++i) {
    const int k = ops[i].kind;
    if ((k == SC_OP_RX || k == SC_OP_RY || k == SC_OP_RZ || k == SC_OP_RZZ) && ops[i].param >= n_params)
      return fail(SC_EINVAL, "op %lld references parameter %d of %lld", (long long)i, ops[i].param,
                  (long long)n_params);
  }
  int rc = c->run(n_qubits, ops, n_ops, nullptr, 0, false, params, n_params);
  if (rc != SC_OK) return rc;
  const int n = c->n;
  const uint64_t full = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
  for (int32_t t = 0; t < n_terms; ++t)
    if ((xmask[t] | zmask[t]) & ~full)
      return fail(SC_EINVAL, "Pauli term %d acts outside the register", t);
  // lambda = H psi (the backward pass starts from it); <H> = Re <lambda | psi>
  const size_t amp = (c->cfg.dtype == SC_C64) ? 8 : 16;
  if ((rc = c->reserve(c->buf_adj_lambda, amp << n, "adjoint lambda")) != SC_OK) return rc;
  if ((rc = reserve_scratch(c, n_params)) != SC_OK) return rc;
  double e = 0.0;
  cudaStream_t s = c->stream;
  const double dim = std::ldexp(1.0, n);
  const int sum_passes = (n_terms + 63) / 64;
  c->mark_begin(KC_ADJOINT, dim * amp * (double)(n_terms + sum_passes + 2), sum_passes + 1);
  cudaError_t ce = cudaSuccess;
  if (n_terms == 0) {
    ce = cudaMemsetAsync(c->buf_adj_lambda.p, 0, amp << n, s);
  } else {
    const int blocks = adjoint_partial_blocks(n, c->sm_count);
    ce = launch_pauli_sum(c->cfg.dtype, c->state.p, c->buf_adj_lambda.p, n, xmask, zmask, coeffs,
                          n_terms, c->sm_count, s);
    if (ce == cudaSuccess)
      ce = launch_inner(c->cfg.dtype, c->buf_adj_lambda.p, c->state.p, n,
                        static_cast<double2*>(c->buf_adj_phi.p), c->sm_count, s);
    std::vector<double2> part(blocks);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(part.data(), c->buf_adj_phi.p, sizeof(double2) * (size_t)blocks,
                           cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    for (int b = 0; b < blocks && ce == cudaSuccess; ++b) e += part[b].x;
  }
  c->mark_end();
  if (ce != cudaSuccess) return fail_cuda(ce, "adjoint H psi");
  if (out_value) *out_value = e;
  c->adj_ops.assign(ops, ops + n_ops);
  c->adj_params.assign(params, params + n_params);
  c->adj_x.assign(xmask, xmask + n_terms);
  c->adj_z.assign(zmask, zmask + n_terms);
  c->adj_c.assign(coeffs, coeffs + n_terms);
  c->adj_ready = true;
  return SC_OK;
}

int32_t sc_adjoint_backward(void* p, double* out_grad, int64_t n_params) {
  Ctx* c = static_cast<Ctx*>(p);
  if (!c || c->magic != Ctx::kMagic) return fail(SC_EINVAL, "invalid context handle");
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(SC_ECUDA, "cudaSetDevice failed");
  if (!c->adj_ready || !c->state_valid)
    return fail(SC_ESTATE, "sc_adjoint_backward needs a preceding sc_adjoint_forward");
  if (n_params != (int64_t)c->adj_params.size() || (n_params > 0 && !out_grad))
    return fail(SC_EINVAL, "gradient buffer must hold %zu entries", c->adj_params.size());
  const int n = c->n;
  const size_t amp = (c->cfg.dtype == SC_C64) ? 8 : 16;
  const int blocks = adjoint_partial_blocks(n, c->sm_count);
  int rc = reserve_scratch(c, n_params);  // lambda and the scratch came with the forward pass
  if (rc != SC_OK) return rc;
  const int max_ctas = c->sm_count * 8;
  double2* partial = static_cast<double2*>(c->buf_adj_phi.p);
  double* grad = static_cast<double*>(c->buf_adj_phi.p) + partial_doubles(c);
  cudaStream_t s = c->stream;
  void* psi = c->state.p;
  void* lam = c->buf_adj_lambda.p;
  const double dim = std::ldexp(1.0, n);
  cudaError_t e = cudaMemsetAsync(grad, 0, sizeof(double) * (size_t)(n_params + 1), s);
  if (e != cudaSuccess) return fail_cuda(e, "gradient init");

  // lambda = H psi was computed by the forward pass
  bool fused = false;
  if (c->adjoint_fused) {
    std::vector<PGate> rev;
    if (reverse_gates(c, rev)) {
      const Plan plan = plan_sweeps(rev, n, reverse_plan_params(c));
      if (adjoint_plan_supported(plan)) {
        fused = true;
        for (size_t k = 0; k < plan.sweeps.size() && e == cudaSuccess; ++k) {
          c->mark_begin(KC_ADJOINT, 4.0 * dim * amp, 2);
          e = launch_adjoint_sweep(c->cfg.dtype, psi, lam, plan, k,
                                   static_cast<double*>(c->buf_adj_phi.p), max_ctas, grad,
                                   c->sm_count, s);
          c->mark_end();
        }
        if (e != cudaSuccess) return fail_cuda(e, "adjoint reverse sweep");
      }
    }
  }
  for (int64_t i = (int64_t)c->adj_ops.size() - 1; i >= 0 && !fused; --i) {
    const sc_op& op = c->adj_ops[i];
    if (op.kind == SC_OP_MEASURE) continue;
    PGate g;
    bool produced = false;
    normalise_op(op, c->adj_params.data(), (int64_t)c->adj_params.size(), &g, &produced);
    if (!produced) continue;
    uint64_t x = 0, z = 0;
    if (op.param >= 0 && generator(op, &x, &z)) {
      c->mark_begin(KC_ADJOINT, 2.0 * dim * amp, 2);
      e = launch_generator_grad(c->cfg.dtype, lam, psi, n, x, z, partial, grad, op.param,
                                c->sm_count, s);
      c->mark_end();
      if (e != cudaSuccess) return fail_cuda(e, "adjoint inner product");
    }
    const PGate inv = invert(g);
    c->mark_begin(KC_ADJOINT, 4.0 * dim * amp, 2);
    e = launch_gate(c->cfg.dtype, psi, n, inv, s);
    if (e == cudaSuccess) e = launch_gate(c->cfg.dtype, lam, n, inv, s);
    c->mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "adjoint un-apply");
  }
  if (n_params > 0 &&
      (e = cudaMemcpyAsync(out_grad, grad, sizeof(double) * (size_t)n_params,
                           cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fail_cuda(e, "gradient download");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail_cuda(e, "sc_adjoint_backward");
  c->collect_timing();
  c->adj_ready = false;
  c->state_valid = false;  // psi has been rewound to the initial state
  return SC_OK;
}

}  // extern "C"
