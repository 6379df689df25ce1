// Host-side inspection of the fusion planner, usable without a GPU.
//
// sc_debug_plan_order reports the order in which the fused kernels apply the
// ops; sc_debug_emulate_sweeps executes a plan on a host complex128 state with
// the same tile / stage / register-bit semantics as k_sweep (the shared-memory
// exchange is a permutation, so a stage is emulated by gathering each thread's
// 2^NR amplitudes straight from the state).  Tests use both to check the planner
// and the plan encoding on CPU.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sc_ctx.h"
#include "sc_sweep.h"

using namespace sc;

namespace {

PlanParams debug_params(int tile, int low, int nr, double budget) {
  PlanParams pp;
  pp.tile_qubits = tile > 0 ? tile : 11;
  pp.low_qubits = low > 0 ? low : 4;
  pp.nr = nr > 0 ? nr : 3;
  pp.budget = budget;
  pp.max_gates = kSweepMaxGates;
  pp.max_pool = kSweepMaxPool;
  if (const char* v = getenv("STATECRAFT_B200_RELAYOUT")) pp.relayout = atoi(v) != 0;
  pp.rot_min_c = 0.05;
  if (const char* v = getenv("STATECRAFT_B200_ROTATION")) pp.rot_min_c = atoi(v) != 0 ? 0.05 : 0.0;
  if (const char* v = getenv("STATECRAFT_B200_PEEPHOLE")) pp.peephole = atoi(v) != 0;
  if (const char* v = getenv("STATECRAFT_B200_ENTRY_FOLD")) pp.entry_fold = atoi(v) != 0;
  return pp;
}

int normalise_all(int n, const sc_op* ops, int64_t n_ops, std::vector<PGate>& out) {
  if (n <= 0 || n > 30) return fail(SC_EINVAL, "debug planner supports 1..30 qubits");
  for (int64_t i = 0; i < n_ops; ++i) {
    PGate g;
    bool produced = false;
    if (!normalise_op(ops[i], nullptr, 0, &g, &produced))
      return fail(SC_EINVAL, "op %lld: unknown kind", (long long)i);
    if (produced) {
      g.op_index = i;
      out.push_back(g);
    }
  }
  return SC_OK;
}

inline uint64_t spread_in(uint32_t x, const SwSweep& sw) {
  uint64_t g = x & ((1u << sw.L) - 1u);
  uint32_t hi = x >> sw.L;
  for (int k = 0; hi; ++k, hi >>= 1)
    if (hi & 1u) g |= 1ULL << sw.hq[k];
  return g;
}

inline uint64_t spread_out(uint32_t x, const SwSweep& sw) {
  uint64_t g = 0;
  for (int p = 0; x; ++p, x >>= 1)
    if (x & 1u) g |= 1ULL << sw.outp[p];
  return g;
}

inline int bitref_h(int ref, uint32_t li, uint64_t base) {
  return ref >= 0 ? (int)((li >> ref) & 1u) : (int)((base >> (-ref - 1)) & 1ULL);
}

struct C {
  double r, i;
};
inline C cm(double br, double bi, C a) { return {br * a.r - bi * a.i, br * a.i + bi * a.r}; }
inline C mac2(const double* m0, C a0, const double* m1, C a1) {
  return {m0[0] * a0.r - m0[1] * a0.i + m1[0] * a1.r - m1[1] * a1.i,
          m0[0] * a0.i + m0[1] * a0.r + m1[0] * a1.i + m1[1] * a1.r};
}

// One sweep: every tile is gathered through the input layout into a buffer indexed
// by tile position, the stages run on it (register j of a thread leaves the stage
// at position l0 | off[perm[j]]), and the tile is scattered through the output
// layout -- the kernel's shared-memory tile, exchanges and final store.
// codes: the Pauli (0 = I, 1 = X, 2 = Y, 3 = Z) of each slot, for plans with slots
void emulate_sweep(double* st, const Plan& plan, const SwSweep& sw,
                   const uint8_t* codes = nullptr) {
  // the kernel sees only the sweep's pool range: a record outside it poisons the state
  for (int gi = sweep_first_gate(plan, sw); gi < plan.stages[sw.s1 - 1].g1; ++gi)
    if (plan.gates[gi].moff < sw.pool0 || plan.gates[gi].moff > sw.pool1) {
      for (uint64_t e = 0; e < 2ULL * (uint64_t)sw.tiles << sw.T; ++e) st[e] = std::nan("");
      return;
    }
  const int NR = sw.nr, NV = 1 << NR;
  const uint32_t tsize = 1u << sw.T;
  const uint32_t threads = 1u << (sw.T - NR);
  std::vector<C> tb(tsize), v(NV);
  std::vector<uint64_t> in_addr(tsize), out_addr(tsize);
  for (uint32_t e = 0; e < tsize; ++e) {
    in_addr[e] = spread_in(e, sw);
    out_addr[e] = spread_out(e, sw);
  }
  std::vector<uint32_t> off(NV);
  for (int64_t t = 0; t < sw.tiles; ++t) {
    uint64_t base = (uint64_t)t << sw.L;
    for (int k = 0; k < sw.h; ++k) {
      const int b = sw.hs[k];
      base = ((base >> b) << (b + 1)) | (base & ((1ULL << b) - 1ULL));
    }
    for (uint32_t e = 0; e < tsize; ++e)
      tb[e] = {st[2 * (base | in_addr[e])], st[2 * (base | in_addr[e]) + 1]};
    for (int s = sw.s0; s < sw.s1; ++s) {
      const SwStage& stg = plan.stages[s];
      for (uint32_t tid = 0; tid < threads; ++tid) {
        uint32_t l0 = tid;
        for (int k = 0; k < NR; ++k) {
          const int b = stg.R[k];
          l0 = ((l0 >> b) << (b + 1)) | (l0 & ((1u << b) - 1u));
        }
        uint32_t xo[16] = {0};  // slot folds: tile-index flips of each register's exit
        for (int j = 0; j < NV; ++j) {
          uint32_t o = 0;
          for (int k = 0; k < NR; ++k)
            if (j & (1 << k)) o |= 1u << stg.R[k];
          off[j] = o;
        }
        // entry folds: register j reads register rperm[j] of the plain read, flipped
        // by rf_d[k] where the condition of the folded record rf_g[k] holds
        int rflip = 0;
        const StageEntry en = plan.entry.empty() ? StageEntry() : plan.entry[s];
        for (int k = 0; k < en.n_rf; ++k) {
          const SwGate& q = plan.gates[en.rf_g[k]];
          if ((base & q.gmask) == q.gmask && (l0 & q.lmask) == q.lmask) rflip ^= en.rf_d[k];
        }
        for (int j = 0; j < NV; ++j) v[j] = tb[l0 | off[en.rperm[j] ^ rflip]];
        for (int gi = stg.g0; gi < stg.g1; ++gi) {
          const SwGate& g = plan.gates[gi];
          if ((base & g.gmask) != g.gmask) continue;
          const double* m = plan.pool.data() + g.moff;
          auto ok = [&](int j) { return ((l0 | off[j]) & g.lmask) == g.lmask; };
          switch (g.kind) {
            case SK_XF:
            case SK_CXF:
              if ((l0 & g.lmask) == g.lmask)
                for (int j = 0; j < NV; ++j)
                  if (g.kind == SK_XF || (j & (1 << g.b))) xo[j] ^= 1u << stg.R[g.a];
              break;
            case SK_X0:
              for (int j = 0; j < NV; ++j)
                if (!(j & (1 << g.a))) std::swap(v[j], v[j | (1 << g.a)]);
              break;
            case SK_PAULI:
            case SK_PAULIF: {  // i^p X^u Z^w over the register bits
              const int code = codes ? codes[g.b] : 0;
              if (code == 0) break;
              int u, w, ph;
              if (g.kind == SK_PAULI) {
                u = code != 3 ? 1 << g.a : 0;
                w = code != 1 ? 1 << g.a : 0;
                ph = code == 2 ? 1 : 0;
              } else {
                u = (int)m[3 * (code - 1)];
                w = (int)m[3 * (code - 1) + 1];
                ph = (int)m[3 * (code - 1) + 2];
              }
              const std::vector<C> src(v);
              for (int j = 0; j < NV; ++j) {
                C x = src[j ^ u];
                if (__builtin_popcount(w & (j ^ u)) & 1) x = {-x.r, -x.i};
                for (int q = 0; q < (ph & 3); ++q) x = {-x.i, x.r};
                v[j] = x;
              }
              break;
            }
            case SK_CX0:
              for (int j = 0; j < NV; ++j)
                if (!(j & (1 << g.a)) && (j & (1 << g.b))) std::swap(v[j], v[j | (1 << g.a)]);
              break;
            case SK_G1:
            case SK_X:
              for (int j = 0; j < NV; ++j) {
                if (j & (1 << g.a)) continue;
                if (!ok(j)) continue;
                const int j1 = j | (1 << g.a);
                if (g.kind == SK_X) {
                  std::swap(v[j], v[j1]);
                } else {
                  const C a0 = v[j], a1 = v[j1];
                  v[j] = mac2(m + 0, a0, m + 2, a1);
                  v[j1] = mac2(m + 4, a0, m + 6, a1);
                }
              }
              break;
            case SK_G2:
              for (int j = 0; j < NV; ++j) {
                if (j & ((1 << g.a) | (1 << g.b))) continue;
                const int idx[4] = {j, j | (1 << g.b), j | (1 << g.a), j | (1 << g.a) | (1 << g.b)};
                C a[4], o[4];
                for (int k = 0; k < 4; ++k) a[k] = v[idx[k]];
                for (int r = 0; r < 4; ++r) {
                  o[r] = {0.0, 0.0};
                  for (int c = 0; c < 4; ++c) {
                    const double mr = m[2 * (4 * r + c)], mi = m[2 * (4 * r + c) + 1];
                    o[r].r += mr * a[c].r - mi * a[c].i;
                    o[r].i += mr * a[c].i + mi * a[c].r;
                  }
                }
                for (int k = 0; k < 4; ++k) v[idx[k]] = o[k];
              }
              break;
            case SK_SWAP:
              for (int j = 0; j < NV; ++j) {
                if (j & ((1 << g.a) | (1 << g.b))) continue;
                std::swap(v[j | (1 << g.a)], v[j | (1 << g.b)]);
              }
              break;
            case SK_D1:
              for (int j = 0; j < NV; ++j) {
                if (!ok(j)) continue;
                const int bit = bitref_h(g.a, l0 | off[j], base);
                v[j] = cm(m[2 * bit], m[2 * bit + 1], v[j]);
              }
              break;
            case SK_D2:
              for (int j = 0; j < NV; ++j) {
                const uint32_t li = l0 | off[j];
                const int k = (bitref_h(g.a, li, base) << 1) | bitref_h(g.b, li, base);
                v[j] = cm(m[2 * k], m[2 * k + 1], v[j]);
              }
              break;
            case SK_G1ALL: {
              const double* mm = m;
              for (int bit = 0; bit < NR; ++bit) {
                if (!((g.a >> bit) & 1)) continue;
                for (int j = 0; j < NV; ++j) {
                  if (j & (1 << bit)) continue;
                  const int j1 = j | (1 << bit);
                  const C a0 = v[j], a1 = v[j1];
                  v[j] = mac2(mm + 0, a0, mm + 2, a1);
                  v[j1] = mac2(mm + 4, a0, mm + 6, a1);
                }
                mm += 8;
              }
              break;
            }
            case SK_G1ALLQ: {
              int bits[8], K = 0;
              for (int bit = 0; bit < NR; ++bit)
                if ((g.a >> bit) & 1) bits[K++] = bit;
              const double* lam = m + 2 * K;
              const double* phi = lam + 2 * ((1 << K) - 1);
              auto subset = [&](int j) {
                int sub = 0;
                for (int k = 0; k < K; ++k) sub |= ((j >> bits[k]) & 1) << k;
                return sub;
              };
              for (int bit = 0; bit < NR; ++bit)  // the record's leading X
                if ((g.b >> bit) & 1)
                  for (int j = 0; j < NV; ++j)
                    if (!(j & (1 << bit))) std::swap(v[j], v[j | (1 << bit)]);
              for (int j = 0; j < NV; ++j)
                if (const int sub = subset(j)) v[j] = cm(lam[2 * (sub - 1)], lam[2 * (sub - 1) + 1], v[j]);
              for (int k = 0; k < K; ++k) {
                // the input table scaled the 1 side by 1 + t^2: two shears
                const double t = m[k], tp = m[K + k];
                for (int j = 0; j < NV; ++j) {
                  if (j & (1 << bits[k])) continue;
                  const int j1 = j | (1 << bits[k]);
                  C a0 = v[j];
                  const C a1 = v[j1];
                  a0 = {std::fma(-tp, a1.r, a0.r), std::fma(-tp, a1.i, a0.i)};
                  v[j] = a0;
                  v[j1] = {std::fma(t, a0.r, a1.r), std::fma(t, a0.i, a1.i)};
                }
              }
              for (int j = 0; j < NV; ++j)
                if (const int sub = subset(j)) v[j] = cm(phi[2 * (sub - 1)], phi[2 * (sub - 1) + 1], v[j]);
              break;
            }
            case SK_DTAB:
              for (int j = 0; j < NV; ++j) v[j] = cm(m[2 * j], m[2 * j + 1], v[j]);
              break;
            case SK_D1R:
              for (int j = 0; j < NV; ++j) {
                const int k = (j >> g.a) & 1;
                v[j] = cm(m[2 * k], m[2 * k + 1], v[j]);
              }
              break;
            case SK_CX:
              for (int j = 0; j < NV; ++j) {
                if ((j & (1 << g.a)) || !(j & (1 << g.b))) continue;
                if ((l0 & g.lmask) != g.lmask) continue;
                std::swap(v[j], v[j | (1 << g.a)]);
              }
              break;
            case SK_DPR:
              for (int j = 0; j < NV; ++j) {
                const int k = ((j >> g.a) ^ (j >> g.b)) & 1;
                v[j] = cm(m[2 * k], m[2 * k + 1], v[j]);
              }
              break;
            case SK_DP:
              for (int j = 0; j < NV; ++j) {
                const uint32_t li = l0 | off[j];
                const int k = bitref_h(g.a, li, base) ^ bitref_h(g.b, li, base);
                v[j] = cm(m[2 * k], m[2 * k + 1], v[j]);
              }
              break;
          }
        }
        // folded permutations: register j leaves the stage as register perm[j]
        for (int j = 0; j < NV; ++j) tb[(l0 | off[stg.perm[j]]) ^ xo[j]] = v[j];
      }
    }
    for (uint32_t e = 0; e < tsize; ++e) {
      const C o = cm(sw.scale_re, sw.scale_im, tb[e]);  // the sweep's rotation-form scalar
      st[2 * (base | out_addr[e])] = o.r;
      st[2 * (base | out_addr[e]) + 1] = o.i;
    }
  }
}

// In-place permutation of physical qubit bits (launch_permute semantics).
void emulate_permute(double* st, int n, const SwPerm& pm) {
  const uint32_t tsize = 1u << pm.nbits;
  std::vector<C> tb(tsize);
  std::vector<uint64_t> addr(tsize);
  for (uint32_t e = 0; e < tsize; ++e) {
    uint64_t g = 0;
    for (int k = 0; k < pm.nbits; ++k)
      if ((e >> k) & 1u) g |= 1ULL << pm.bits[k];
    addr[e] = g;
  }
  const int64_t tiles = 1LL << (n - pm.nbits);
  for (int64_t t = 0; t < tiles; ++t) {
    uint64_t base = (uint64_t)t;
    for (int k = 0; k < pm.nbits; ++k) {
      const int b = pm.bits[k];
      base = ((base >> b) << (b + 1)) | (base & ((1ULL << b) - 1ULL));
    }
    for (uint32_t e = 0; e < tsize; ++e)
      tb[e] = {st[2 * (base | addr[e])], st[2 * (base | addr[e]) + 1]};
    for (uint32_t o = 0; o < tsize; ++o) {
      uint32_t i = 0;
      for (int k = 0; k < pm.nbits; ++k)
        if ((o >> k) & 1u) i |= 1u << pm.src[k];
      st[2 * (base | addr[o])] = tb[i].r;
      st[2 * (base | addr[o]) + 1] = tb[i].i;
    }
  }
}

}  // namespace

extern "C" {

int32_t sc_debug_entry_folds(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                             int32_t low_qubits, int32_t nr, double budget, int64_t* stats) {
  std::vector<PGate> gates;
  int rc = normalise_all(n, ops, n_ops, gates);
  if (rc != SC_OK) return rc;
  if (!stats) return fail(SC_EINVAL, "stats[3] is required");
  Plan plan = plan_sweeps(gates, n, debug_params(tile_qubits, low_qubits, nr, budget));
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  stats[0] = (int64_t)plan.stages.size();
  stats[1] = stats[2] = 0;
  for (size_t s = 0; s < plan.entry.size(); ++s) {
    stats[1] += plan.stages[s].g0 - plan.entry[s].g_start;
    stats[2] += plan.entry[s].n_rf;
  }
  return SC_OK;
}

int32_t sc_debug_plan_order(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                            int32_t low_qubits, int32_t nr, double budget, int64_t* order,
                            int64_t* n_sweeps, int64_t* n_stages, int64_t* n_relayouts,
                            int64_t* n_restores) {
  std::vector<PGate> gates;
  int rc = normalise_all(n, ops, n_ops, gates);
  if (rc != SC_OK) return rc;
  Plan plan = plan_sweeps(gates, n, debug_params(tile_qubits, low_qubits, nr, budget));
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  if (order)
    for (size_t i = 0; i < plan.gate_ops.size(); ++i) order[i] = plan.gate_ops[i];
  if (n_sweeps) *n_sweeps = (int64_t)plan.sweeps.size();
  if (n_stages) *n_stages = (int64_t)plan.stages.size();
  if (n_relayouts) {
    *n_relayouts = 0;
    for (const SwSweep& sw : plan.sweeps) *n_relayouts += sw.relayout ? 1 : 0;
  }
  if (n_restores) *n_restores = (int64_t)plan.restore.size();
  return (int32_t)plan.gate_ops.size();
}

int32_t sc_debug_emulate_sweeps(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                                int32_t low_qubits, int32_t nr, double budget, double* state) {
  std::vector<PGate> gates;
  int rc = normalise_all(n, ops, n_ops, gates);
  if (rc != SC_OK) return rc;
  if (!state) return fail(SC_EINVAL, "state is null");
  Plan plan = plan_sweeps(gates, n, debug_params(tile_qubits, low_qubits, nr, budget));
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  for (const SwSweep& sw : plan.sweeps) emulate_sweep(state, plan, sw);
  for (const SwPerm& pm : plan.restore) emulate_permute(state, n, pm);
  return (int32_t)plan.sweeps.size();
}

int32_t sc_debug_emulate_slots(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                               int32_t low_qubits, int32_t nr, double budget,
                               const int64_t* slot_after, const int32_t* slot_qubit,
                               int64_t n_slots, const uint8_t* paulis, double* state) {
  if (!state || (n_slots > 0 && (!slot_after || !slot_qubit || !paulis)))
    return fail(SC_EINVAL, "null argument");
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
    for (; next < n_slots && slot_after[next] == i; ++next) {
      if (slot_qubit[next] < 0 || slot_qubit[next] >= n || paulis[next] > 3)
        return fail(SC_EINVAL, "slot %lld: bad qubit or Pauli", (long long)next);
      PGate sg;
      std::memset(&sg, 0, sizeof sg);
      sg.kind = PK_PAULI;
      sg.q0 = slot_qubit[next];
      sg.q1 = (int32_t)next;
      sg.op_index = i;
      gates.push_back(sg);
    }
  }
  if (next != n_slots) return fail(SC_EINVAL, "slot_after must be sorted op indices");
  PlanParams pp = debug_params(tile_qubits, low_qubits, nr, budget);
  pp.relayout = false;
  Plan plan = plan_sweeps(gates, n, pp);
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  for (const SwSweep& sw : plan.sweeps) emulate_sweep(state, plan, sw, paulis);
  return (int32_t)plan.sweeps.size();
}

int32_t sc_debug_check_exchanges(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                                 int32_t low_qubits, int32_t nr, int32_t dtype, int64_t* stats) {
  std::vector<PGate> gates;
  int rc = normalise_all(n, ops, n_ops, gates);
  if (rc != SC_OK) return rc;
  if (!stats) return fail(SC_EINVAL, "stats is null");
  if (dtype != SC_C64 && dtype != SC_C128) return fail(SC_EINVAL, "dtype must be SC_C64 or SC_C128");
  PlanParams pp = debug_params(tile_qubits, low_qubits, nr, -1.0);
  pp.relayout = false;
  Plan plan = plan_sweeps(gates, n, pp);
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  if (!check_exchange_tables(plan, dtype, stats))
    return fail(SC_ESTATE, "inconsistent shared-memory exchange tables");
  return (int32_t)plan.sweeps.size();
}

int32_t sc_debug_check_tile_tensors(int32_t n, const sc_op* ops, int64_t n_ops,
                                    int32_t tile_qubits, int32_t low_qubits, int32_t nr,
                                    int32_t dtype, int64_t batch, int64_t* stats) {
  std::vector<PGate> gates;
  int rc = normalise_all(n, ops, n_ops, gates);
  if (rc != SC_OK) return rc;
  if (!stats) return fail(SC_EINVAL, "stats is null");
  if (dtype != SC_C64 && dtype != SC_C128) return fail(SC_EINVAL, "dtype must be SC_C64 or SC_C128");
  if (batch < 1) return fail(SC_EINVAL, "batch must be positive");
  PlanParams pp = debug_params(tile_qubits, low_qubits, nr, -1.0);
  Plan plan = plan_sweeps(gates, n, pp);
  if (!plan.ok) return fail(SC_ECUDA, "fusion planner could not stage every gate");
  if (!check_tile_tensors(plan, dtype, batch, stats))
    return fail(SC_ESTATE, "a tile tensor copy does not match the sweep's tile enumeration");
  return (int32_t)plan.sweeps.size();
}

}  // extern "C"
