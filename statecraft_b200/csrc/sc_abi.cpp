// C ABI entry points: context management, validation mirroring the reference
// engine's exceptions, the op loop (fused or per gate), noise, measurement and
// expectation values.  All device work runs on the context's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "sc_ctx.h"
#include "sc_sweep.h"

namespace sc {

thread_local std::string tl_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  tl_error = buf;
  return code;
}

int fail_cuda(cudaError_t e, const char* where) {
  return fail(e == cudaErrorMemoryAllocation ? SC_ENOMEM : SC_ECUDA, "%s: %s (%s)", where,
              cudaGetErrorString(e), cudaGetErrorName(e));
}

const char* kernel_class_name(int cls) {
  static const char* names[KC_COUNT] = {"sweep",  "gate_dense", "gate_perm", "gate_diag",
                                        "init",   "probabilities", "sample",  "noise",
                                        "expect", "adjoint",    "batch",   "permute",
                                        "block"};
  return (cls >= 0 && cls < KC_COUNT) ? names[cls] : "unknown";
}

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
int Ctx::reserve(DevBuf& b, size_t bytes, const char* what) {
  if (bytes <= b.cap) return SC_OK;
  const size_t other = allocated - b.cap;
  if (cfg.device_mem_limit > 0 && other + bytes > (size_t)cfg.device_mem_limit)
    return fail(SC_ENOMEM, "device memory limit of %lld bytes exceeded allocating %s (%zu bytes)",
                (long long)cfg.device_mem_limit, what, bytes);
  if (b.p) {
    cudaStreamSynchronize(stream);
    cudaFree(b.p);
    allocated -= b.cap;
    b.p = nullptr;
    b.cap = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(SC_ENOMEM, "cudaMalloc of %zu bytes for %s failed: %s", bytes, what,
                cudaGetErrorString(e));
  }
  b.cap = bytes;
  allocated += bytes;
  return SC_OK;
}

void Ctx::release(DevBuf& b) {
  if (b.p) {
    cudaFree(b.p);
    allocated -= b.cap;
  }
  b.p = nullptr;
  b.cap = 0;
}

// ---------------------------------------------------------------------------
// timing
// ---------------------------------------------------------------------------
void Ctx::mark_begin(int cls, double bytes, int kernels) {
  stats_launch[cls] += kernels;
  if (!cfg.timing) return;
  Timed t;
  t.cls = cls;
  t.bytes = bytes;
  t.a = get_event();
  t.b = get_event();
  cudaEventRecord(t.a, stream);
  pending.push_back(t);
}

void Ctx::mark_end() {
  if (!cfg.timing || pending.empty()) return;
  cudaEventRecord(pending.back().b, stream);
}

cudaEvent_t Ctx::get_event() {
  if (event_pool_next < event_pool.size()) return event_pool[event_pool_next++];
  cudaEvent_t e;
  cudaEventCreate(&e);
  event_pool.push_back(e);
  ++event_pool_next;
  return e;
}

void Ctx::collect_timing() {
  if (!cfg.timing) return;
  for (const Timed& t : pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      stats_ms[t.cls] += ms;
      stats_bytes[t.cls] += t.bytes;
    }
  }
  cudaGetLastError();
  pending.clear();
  event_pool_next = 0;
}

}  // namespace sc

using namespace sc;

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
namespace {

Ctx* as_ctx(void* p) { return static_cast<Ctx*>(p); }

int check_ctx(Ctx* c) {
  if (!c || c->magic != Ctx::kMagic) return fail(SC_EINVAL, "invalid context handle");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  return SC_OK;
}

bool in_range(int q, int n) { return q >= 0 && q < n; }

bool is_unitary(int kind) {
  switch (kind) {
    case SC_OP_SINGLE: case SC_OP_CNOT: case SC_OP_TWO: case SC_OP_DIAG2: case SC_OP_SWAP:
    case SC_OP_MULTI: case SC_OP_RX: case SC_OP_RY: case SC_OP_RZ: case SC_OP_RZZ:
      return true;
    default:
      return false;
  }
}

// Mirrors the Operation record validation (QuantumCircuit.java:362-574) and the
// engine's limits and measurement rule (StatevectorEngine.java:90-151, 169-174).
int validate_ops(int n, const sc_op* ops, int64_t n_ops, int max_qubits) {
  if (n <= 0) return fail(SC_EINVAL, "qubitCount must be positive");
  if (n > max_qubits)
    return fail(SC_EUNSUPPORTED, "statevector engine supports up to %d qubits in dense mode, got %d",
                max_qubits, n);
  if (n_ops < 0 || (n_ops > 0 && !ops)) return fail(SC_EINVAL, "invalid op array");
  const uint64_t full = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
  bool measured = false;
  for (int64_t i = 0; i < n_ops; ++i) {
    const sc_op& op = ops[i];
    if (op.kind == SC_OP_MEASURE) {
      if (op.mask == 0) return fail(SC_EINVAL, "op %lld: at least one qubit must be measured", (long long)i);
      if (op.mask & ~full) return fail(SC_EINVAL, "op %lld: measured qubit out of range", (long long)i);
      measured = true;
      continue;
    }
    if (!is_unitary(op.kind)) return fail(SC_EINVAL, "op %lld: unknown operation kind %d", (long long)i, op.kind);
    if (measured)
      return fail(SC_EUNSUPPORTED, "Unitary operations cannot follow measurement operations in the circuit");
    switch (op.kind) {
      case SC_OP_SINGLE: case SC_OP_RX: case SC_OP_RY: case SC_OP_RZ:
        if (!in_range(op.q0, n)) return fail(SC_EINVAL, "target qubit out of range: %d", op.q0);
        break;
      case SC_OP_CNOT:
        if (!in_range(op.q0, n)) return fail(SC_EINVAL, "control qubit out of range: %d", op.q0);
        if (!in_range(op.q1, n)) return fail(SC_EINVAL, "target qubit out of range: %d", op.q1);
        if (op.q0 == op.q1) return fail(SC_EINVAL, "control and target qubits must differ");
        break;
      case SC_OP_TWO: case SC_OP_DIAG2: case SC_OP_SWAP: case SC_OP_RZZ:
        if (!in_range(op.q0, n)) return fail(SC_EINVAL, "first qubit out of range: %d", op.q0);
        if (!in_range(op.q1, n)) return fail(SC_EINVAL, "second qubit out of range: %d", op.q1);
        if (op.q0 == op.q1) return fail(SC_EINVAL, "qubits must be distinct");
        break;
      case SC_OP_MULTI:
        if (!in_range(op.q0, n)) return fail(SC_EINVAL, "target qubit out of range: %d", op.q0);
        if (op.mask == 0) return fail(SC_EINVAL, "at least one control qubit is required");
        if (op.mask & ~full) return fail(SC_EINVAL, "control qubit out of range");
        if ((op.mask >> op.q0) & 1ULL) return fail(SC_EINVAL, "control and target qubits must differ");
        break;
    }
  }
  return SC_OK;
}

int validate_channels(const std::vector<sc_channel>& ch, const sc_op* ops, int64_t n_ops, int n) {
  int64_t prev = -1;
  for (size_t k = 0; k < ch.size(); ++k) {
    const sc_channel& c = ch[k];
    if (c.after_op < 0 || c.after_op >= n_ops)
      return fail(SC_EINVAL, "noise record %zu follows op %lld outside the circuit", k, (long long)c.after_op);
    if (c.after_op < prev) return fail(SC_EINVAL, "noise records must be sorted by after_op");
    prev = c.after_op;
    if (!is_unitary(ops[c.after_op].kind))
      return fail(SC_EINVAL, "noise record %zu follows a non-unitary op", k);
    if (c.target < 0 || c.target >= n)
      return fail(SC_EINVAL, "noise channel qubit out of range: %d", c.target);
    if (c.n_kraus < 1 || c.n_kraus > SC_MAX_KRAUS)
      return fail(SC_EINVAL, "noise record %zu: n_kraus must be in [1, %d]", k, SC_MAX_KRAUS);
  }
  return SC_OK;
}

uint64_t fresh_seed() {
  std::random_device rd;
  uint64_t s = ((uint64_t)rd() << 32) ^ rd();
  s ^= (uint64_t)std::chrono::high_resolution_clock::now().time_since_epoch().count();
  return s;
}

}  // namespace

// ---------------------------------------------------------------------------
// the op loop
// ---------------------------------------------------------------------------
namespace sc {

int check_context(void* p) { return check_ctx(as_ctx(p)); }
int validate_circuit(int n, const sc_op* ops, int64_t n_ops, int max_qubits) {
  return validate_ops(n, ops, n_ops, max_qubits);
}
int validate_noise(const std::vector<sc_channel>& ch, const sc_op* ops, int64_t n_ops, int n) {
  return validate_channels(ch, ops, n_ops, n);
}

PlanParams Ctx::plan_params() const {
  PlanParams pp;
  const bool c64 = cfg.dtype == SC_C64;
  // 2048-amplitude tiles, 16 amplitudes per thread; no per-sweep FMA cap (the
  // sweeps are issue-bound, so fewer, fuller sweeps save HBM passes for free)
  pp.tile_qubits = cfg.tile_qubits > 0 ? cfg.tile_qubits : 11;
  pp.low_qubits = low_qubits > 0 ? low_qubits : (c64 ? 5 : 4);
  pp.nr = nr > 0 ? nr : 4;
  pp.budget = cfg.sweep_budget > 0 ? (double)cfg.sweep_budget : -1.0;
  pp.max_gates = kSweepMaxGates;
  pp.max_pool = kSweepMaxPool;
  pp.relayout = relayout;
  // rotation form for 1-qubit unitaries: |u00| >= 0.05 (c128) / 0.25 (c64) keeps
  // t <= 20 / 4; the scalar floor keeps the stored amplitudes below 2^400 (c128)
  // or 2^60 (c64), and the scalar a sweep applies a normal number
  pp.rot_min_c = rotation ? (c64 ? 0.25 : 0.05) : 0.0;
  pp.scale_floor = c64 ? 0x1p-30 : 0x1p-200;
  pp.peephole = peephole;
  pp.entry_fold = entry_fold;
  return pp;
}

int Ctx::apply_gates(const std::vector<PGate>& gates) {
  if (gates.empty()) return SC_OK;
  const double amp_bytes = (cfg.dtype == SC_C64) ? 8.0 : 16.0;
  const double dim = std::ldexp(1.0, n);
  if (!cfg.fusion) {
    for (const PGate& g : gates) {
      int cls = (g.kind == PK_DENSE1 || g.kind == PK_DENSE2) ? KC_GATE_DENSE
                : (g.kind == PK_X || g.kind == PK_SWAP)      ? KC_GATE_PERM
                                                             : KC_GATE_DIAG;
      mark_begin(cls, 2.0 * dim * amp_bytes);
      cudaError_t e = launch_gate(cfg.dtype, state.p, n, g, stream);
      mark_end();
      if (e != cudaSuccess) return fail_cuda(e, "gate kernel");
      ++plan_gates;
    }
    return SC_OK;
  }
  if (dense_block_cost > 0.0 && cfg.dtype == SC_C128) {
    // runs of gates on at most 5 qubits heavy enough for a dense block go to the
    // tensor-core kernel; the rest is planned into sweeps run by run
    std::vector<DenseBlock> blocks;
    std::vector<GateRun> runs = cut_dense_blocks(gates, n, dense_block_cost, &blocks);
    if (!blocks.empty()) {
      size_t elems = 0;
      for (const DenseBlock& b : blocks) elems += b.u.size();
      int rc = reserve(buf_block, sizeof(double) * elems, "dense block matrices");
      if (rc != SC_OK) return rc;
      std::vector<double> host;
      host.reserve(elems);
      std::vector<size_t> offs;
      for (const DenseBlock& b : blocks) {
        offs.push_back(host.size());
        host.insert(host.end(), b.u.begin(), b.u.end());
      }
      cudaError_t e = cudaMemcpyAsync(buf_block.p, host.data(), sizeof(double) * elems,
                                      cudaMemcpyHostToDevice, stream);
      if (e != cudaSuccess) return fail_cuda(e, "dense block upload");
      for (const GateRun& r : runs) {
        if ((rc = apply_sweeps(r.gates)) != SC_OK) return rc;
        if (r.block < 0) continue;
        const DenseBlock& b = blocks[(size_t)r.block];
        mark_begin(KC_BLOCK, 2.0 * dim * amp_bytes);
        e = launch_block(state.p, n, b.args, static_cast<const double*>(buf_block.p) + offs[(size_t)r.block],
                         sm_count, stream);
        mark_end();
        if (e != cudaSuccess) return fail_cuda(e, "dense block kernel");
        ++plan_sweeps_count;
        ++plan_blocks;
        plan_gates += b.n_gates;
      }
      // the host copy must outlive the upload
      if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "dense blocks");
      return SC_OK;
    }
  }
  return apply_sweeps(gates);
}

namespace {

bool same_plan_params(const PlanParams& a, const PlanParams& b) {
  return a.tile_qubits == b.tile_qubits && a.low_qubits == b.low_qubits && a.nr == b.nr &&
         a.budget == b.budget && a.max_gates == b.max_gates && a.max_pool == b.max_pool &&
         a.relayout == b.relayout && a.rot_min_c == b.rot_min_c &&
         a.scale_floor == b.scale_floor && a.peephole == b.peephole &&
         a.entry_fold == b.entry_fold && a.phase_free == b.phase_free;
}

bool same_gates(const std::vector<PGate>& a, const std::vector<PGate>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i) {
    const PGate &x = a[i], &y = b[i];
    if (x.kind != y.kind || x.q0 != y.q0 || x.q1 != y.q1 || x.cmask != y.cmask ||
        x.op_index != y.op_index || std::memcmp(x.m, y.m, sizeof x.m) != 0)
      return false;
  }
  return true;
}

}  // namespace

int Ctx::apply_sweeps(const std::vector<PGate>& gates) {
  if (gates.empty()) return SC_OK;
  const double amp_bytes = (cfg.dtype == SC_C64) ? 8.0 : 16.0;
  const double dim = std::ldexp(1.0, n);
  const PlanParams pp = plan_params();
  if (!(plan_cache_valid && plan_cache_n == n && same_plan_params(plan_cache_pp, pp) &&
        same_gates(plan_cache_gates, gates))) {
    plan_cache_valid = false;
    plan_cache = plan_sweeps(gates, n, pp);
    plan_cache_gates = gates;
    plan_cache_n = n;
    plan_cache_pp = pp;
    plan_cache_valid = plan_cache.ok;
  }
  const Plan& plan = plan_cache;
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  for (size_t k = 0; k < plan.sweeps.size(); ++k) {
    mark_begin(KC_SWEEP, 2.0 * dim * amp_bytes);
    cudaError_t e = launch_sweep(cfg.dtype, state.p, plan, k, static_cast<int*>(buf_err.p),
                                 sm_count, stream);
    mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "sweep kernel");
  }
  for (const SwPerm& pm : plan.restore) {
    mark_begin(KC_PERMUTE, 2.0 * dim * amp_bytes);
    cudaError_t e = launch_permute(cfg.dtype, state.p, n, pm, sm_count, stream);
    mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "layout restore kernel");
  }
  plan_sweeps_count += (int64_t)plan.sweeps.size();
  plan_gates += plan.n_gates;
  plan_stages += (int64_t)plan.stages.size();
  return SC_OK;
}

int Ctx::ensure_state(int nq) {
  const size_t amp = (cfg.dtype == SC_C64) ? 8 : 16;
  const size_t bytes = amp << nq;
  int rc = reserve(state, bytes, "state vector");
  if (rc != SC_OK) return rc;
  n = nq;
  return SC_OK;
}

int Ctx::run(int nq, const sc_op* ops, int64_t n_ops, const double* init, uint64_t basis,
             bool has_basis, const double* params, int64_t n_params) {
  state_valid = false;
  adj_ready = false;  // a pending adjoint pair refers to the state this run replaces
  // a noise schedule applies to one run only
  std::vector<sc_channel> noise_sched;
  noise_sched.swap(this->noise);
  const std::vector<sc_channel>& noise = noise_sched;
  int rc = validate_ops(nq, ops, n_ops, max_qubits);
  if (rc != SC_OK) return rc;
  if (has_basis && nq < 64 && (basis >> nq) != 0)
    return fail(SC_EINVAL, "basis-state qubit out of range");
  if ((rc = validate_channels(noise, ops, n_ops, nq)) != SC_OK) return rc;
  if ((rc = ensure_state(nq)) != SC_OK) return rc;
  if ((rc = reserve(buf_err, 16, "error flag")) != SC_OK) return rc;
  cudaMemsetAsync(buf_err.p, 0, 16, stream);
  plan_sweeps_count = plan_gates = plan_stages = plan_blocks = 0;

  // state preparation (populateFromState / resetBasisState / resetZeroState)
  const double dim = std::ldexp(1.0, nq);
  const double amp_bytes = (cfg.dtype == SC_C64) ? 8.0 : 16.0;
  if (init) {
    const size_t bytes = (size_t)16 << nq;
    cudaError_t e;
    if (cfg.dtype == SC_C64) {
      if ((rc = reserve(buf_convert, bytes, "initial-state staging")) != SC_OK) return rc;
      if ((e = cudaMemcpyAsync(buf_convert.p, init, bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return fail_cuda(e, "initial state upload");
      mark_begin(KC_INIT, dim * (16.0 + amp_bytes));
      e = launch_convert_in(cfg.dtype, state.p, static_cast<const double*>(buf_convert.p),
                            (int64_t)1 << nq, stream);
      mark_end();
    } else {
      e = cudaMemcpyAsync(state.p, init, bytes, cudaMemcpyHostToDevice, stream);
    }
    if (e != cudaSuccess) return fail_cuda(e, "initial state upload");
  } else {
    mark_begin(KC_INIT, dim * amp_bytes);
    cudaError_t e = launch_init_basis(cfg.dtype, state.p, nq, has_basis ? basis : 0ULL, stream);
    mark_end();
    if (e != cudaSuccess) return fail_cuda(e, "state init");
  }

  // measured-qubit default (resolveMeasuredQubits)
  uint64_t mmask = 0;
  bool any_measure = false;
  for (int64_t i = 0; i < n_ops; ++i)
    if (ops[i].kind == SC_OP_MEASURE) {
      mmask |= ops[i].mask;
      any_measure = true;
    }
  default_measured.clear();
  for (int q = 0; q < nq; ++q)
    if (!any_measure || ((mmask >> q) & 1ULL)) default_measured.push_back(q);

  // noise bookkeeping
  if (!noise.empty()) {
    if ((rc = reserve(buf_noise_state, sizeof(NoiseDevState), "noise state")) != SC_OK) return rc;
    if ((rc = reserve(buf_noise_partial,
                      sizeof(double) * SC_MAX_KRAUS * (size_t)noise_grid(nq, sm_count),
                      "noise partials")) != SC_OK)
      return rc;
    cudaMemsetAsync(buf_noise_state.p, 0, sizeof(NoiseDevState), stream);
  }

  // op loop: gates between noise points are planned together
  std::vector<PGate> seg;
  size_t next_ch = 0;
  uint64_t draw = 0;
  for (int64_t i = 0; i < n_ops; ++i) {
    PGate g;
    bool produced = false;
    if (!normalise_op(ops[i], params, n_params, &g, &produced))
      return fail(SC_EINVAL, "op %lld: cannot normalise", (long long)i);
    if (produced) {
      g.op_index = i;
      seg.push_back(g);
    }
    if (next_ch < noise.size() && noise[next_ch].after_op == i) {
      if ((rc = apply_gates(seg)) != SC_OK) return rc;
      seg.clear();
      while (next_ch < noise.size() && noise[next_ch].after_op == i) {
        const sc_channel& c = noise[next_ch];
        KrausArgs ka;
        std::memset(&ka, 0, sizeof ka);
        ka.nk = c.n_kraus;
        ka.target = c.target;
        for (int k = 0; k < c.n_kraus; ++k) std::memcpy(ka.k[k], c.kraus[k], 8 * sizeof(double));
        mark_begin(KC_NOISE, 3.0 * dim * amp_bytes, 3);
        cudaError_t e = launch_kraus_channel(cfg.dtype, state.p, nq, ka, noise_seed, draw,
                                             static_cast<double*>(buf_noise_partial.p),
                                             static_cast<NoiseDevState*>(buf_noise_state.p),
                                             sm_count, stream);
        mark_end();
        if (e != cudaSuccess) return fail_cuda(e, "noise kernel");
        ++draw;
        ++next_ch;
      }
    }
  }
  if ((rc = apply_gates(seg)) != SC_OK) return rc;

  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail_cuda(e, "sc_run");
  collect_timing();
  int err_flag = 0;
  if ((e = cudaMemcpy(&err_flag, buf_err.p, sizeof err_flag, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "error flag");
  if (err_flag) return fail(SC_ETIMEOUT, "sweep kernel timed out waiting for a bulk copy");
  if (!noise.empty()) {
    NoiseDevState ns;
    e = cudaMemcpy(&ns, buf_noise_state.p, offsetof(NoiseDevState, choices), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail_cuda(e, "noise status");
    if (ns.status == kNoiseBadWeight || ns.status == kNoiseBadTotal)
      return fail(SC_ESTATE, "invalid Kraus branch weights at noise draw %llu",
                  (unsigned long long)ns.bad_draw);
    if (ns.status == kNoiseBadNorm)
      return fail(SC_ESTATE, "state collapsed to invalid norm after Kraus application");
  }
  state_valid = true;
  return SC_OK;
}

}  // namespace sc

// ---------------------------------------------------------------------------
// exported entry points
// ---------------------------------------------------------------------------
extern "C" {

int32_t sc_version(void) { return SC_ABI_VERSION; }

const char* sc_last_error(void) { return tl_error.c_str(); }

int32_t sc_create(int32_t device, const sc_config* cfg, void** out_ctx) {
  if (!out_ctx) return fail(SC_EINVAL, "out_ctx is null");
  *out_ctx = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDeviceCount");
  if (device < 0 || device >= count)
    return fail(SC_EINVAL, "device %d out of range (%d devices)", device, count);
  if ((e = cudaSetDevice(device)) != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
  Ctx* c = new Ctx();
  c->device = device;
  if (cfg) c->cfg = *cfg;
  else {
    std::memset(&c->cfg, 0, sizeof c->cfg);
    c->cfg.fusion = 1;
  }
  if (c->cfg.dtype != SC_C128 && c->cfg.dtype != SC_C64) {
    delete c;
    return fail(SC_EINVAL, "dtype must be SC_C128 or SC_C64");
  }
  c->max_qubits = c->cfg.max_qubits > 0 ? c->cfg.max_qubits : SC_DEFAULT_MAX_QUBITS;
  if (c->max_qubits > SC_DEFAULT_MAX_QUBITS) c->max_qubits = SC_DEFAULT_MAX_QUBITS;
  if ((e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete c;
    return fail_cuda(e, "sc_create");
  }
  if (const char* v = getenv("STATECRAFT_B200_LOW_QUBITS")) c->low_qubits = atoi(v);
  if (const char* v = getenv("STATECRAFT_B200_NR")) c->nr = atoi(v);
  if (const char* v = getenv("STATECRAFT_B200_RELAYOUT")) c->relayout = atoi(v) != 0;
  if (const char* v = getenv("STATECRAFT_B200_ROTATION")) c->rotation = atoi(v) != 0;
  if (const char* v = getenv("STATECRAFT_B200_PEEPHOLE")) c->peephole = atoi(v) != 0;
  if (const char* v = getenv("STATECRAFT_B200_ENTRY_FOLD")) c->entry_fold = atoi(v) != 0;
  if (const char* v = getenv("STATECRAFT_B200_ADJOINT_FUSED")) c->adjoint_fused = atoi(v) != 0;
  // minimum sweep-path cost of a dense block (FMA per amplitude); 0 turns blocks off
  if (const char* v = getenv("STATECRAFT_B200_DENSE_BLOCKS")) c->dense_block_cost = atof(v);
  *out_ctx = c;
  return SC_OK;
}

int32_t sc_destroy(void* p) {
  Ctx* c = as_ctx(p);
  if (!c) return SC_OK;
  if (c->magic != Ctx::kMagic) return fail(SC_EINVAL, "invalid context handle");
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (void* b : c->qaoa_batches) qaoa_batch_free(b);
  c->qaoa_batches.clear();
  traj_cache_free(c->traj_cache);
  c->traj_cache = nullptr;
  c->release_all();
  for (cudaEvent_t ev : c->event_pool) cudaEventDestroy(ev);
  cudaStreamDestroy(c->stream);
  c->magic = 0;
  delete c;
  return SC_OK;
}

int32_t sc_set_noise(void* p, const sc_channel* ch, int64_t n, uint64_t seed, int32_t has_seed) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  if (n < 0 || (n > 0 && !ch)) return fail(SC_EINVAL, "invalid noise record array");
  c->noise.assign(ch, ch + n);
  c->noise_seed = has_seed ? seed : fresh_seed();
  return SC_OK;
}

int32_t sc_run(void* p, int32_t n_qubits, const sc_op* ops, int64_t n_ops,
               const double* init_state, uint64_t basis_mask, int32_t has_basis) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  return c->run(n_qubits, ops, n_ops, init_state, basis_mask, has_basis != 0, nullptr, 0);
}

int32_t sc_get_state(void* p, double* out, int64_t n_doubles) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  if (!c->state_valid) return fail(SC_ESTATE, "no state: sc_run has not completed");
  if (!out || n_doubles != ((int64_t)2 << c->n))
    return fail(SC_EINVAL, "output must hold 2^(n+1) = %lld doubles", (long long)((int64_t)2 << c->n));
  const size_t bytes = (size_t)16 << c->n;
  cudaError_t e;
  if (c->cfg.dtype == SC_C64) {
    if ((rc = c->reserve(c->buf_convert, bytes, "state staging")) != SC_OK) return rc;
    if ((e = launch_convert_out(c->cfg.dtype, c->state.p, static_cast<double*>(c->buf_convert.p),
                                (int64_t)1 << c->n, c->stream)) != cudaSuccess)
      return fail_cuda(e, "state conversion");
    e = cudaMemcpyAsync(out, c->buf_convert.p, bytes, cudaMemcpyDeviceToHost, c->stream);
  } else {
    e = cudaMemcpyAsync(out, c->state.p, bytes, cudaMemcpyDeviceToHost, c->stream);
  }
  if (e != cudaSuccess) return fail_cuda(e, "state download");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail_cuda(e, "state download");
  return SC_OK;
}

int32_t sc_default_measured_qubits(void* p, int32_t* out, int32_t cap) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  if (!c->state_valid) return fail(SC_ESTATE, "no state: sc_run has not completed");
  const int32_t count = (int32_t)c->default_measured.size();
  for (int32_t k = 0; k < count && k < cap && out; ++k) out[k] = c->default_measured[k];
  return count;
}

int32_t sc_sample(void* p, const int32_t* qubits, int32_t m, int64_t shots, uint64_t seed,
                  int32_t has_seed, const double* uniforms, int32_t* outcomes) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  return c->sample(qubits, m, shots, has_seed ? seed : fresh_seed(), uniforms, outcomes);
}

int32_t sc_probabilities(void* p, const int32_t* qubits, int32_t m, double* out) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  return c->probabilities(qubits, m, out);
}

int32_t sc_expect_pauli(void* p, int32_t n_terms, const uint64_t* xmask, const uint64_t* zmask,
                        const double* coeffs, double* out_value) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  if (!c->state_valid) return fail(SC_ESTATE, "no state: sc_run has not completed");
  std::vector<double> terms;
  if ((rc = c->pauli_terms(n_terms, xmask, zmask, terms)) != SC_OK) return rc;
  double total = 0.0;
  for (int32_t t = 0; t < n_terms; ++t) total += coeffs[t] * terms[t];
  if (out_value) *out_value = total;
  return SC_OK;
}

int32_t sc_kernel_stats(void* p, int64_t* launches, double* ms, double* bytes, int32_t cap) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  for (int k = 0; k < KC_COUNT && k < cap; ++k) {
    if (launches) launches[k] = c->stats_launch[k];
    if (ms) ms[k] = c->stats_ms[k];
    if (bytes) bytes[k] = c->stats_bytes[k];
  }
  return KC_COUNT;
}

const char* sc_kernel_class_name(int32_t cls) { return kernel_class_name(cls); }

int32_t sc_reset_kernel_stats(void* p) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  for (int k = 0; k < KC_COUNT; ++k) {
    c->stats_launch[k] = 0;
    c->stats_ms[k] = 0.0;
    c->stats_bytes[k] = 0.0;
  }
  return SC_OK;
}

void* sc_stream(void* p) {
  Ctx* c = as_ctx(p);
  if (!c || c->magic != Ctx::kMagic) return nullptr;
  return static_cast<void*>(c->stream);
}

int32_t sc_last_plan_stats(void* p, int64_t* sweeps, int64_t* gates, int64_t* stages) {
  Ctx* c = as_ctx(p);
  int rc = check_ctx(c);
  if (rc != SC_OK) return rc;
  if (sweeps) *sweeps = c->plan_sweeps_count;
  if (gates) *gates = c->plan_gates;
  if (stages) *stages = c->plan_stages;
  return SC_OK;
}

}  // extern "C"
