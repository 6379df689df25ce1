// Gate normalisation and the fusion planner (host side).
//
// The reference engine applies one full-state sweep per operation
// (StatevectorEngine.java:90-151).  Here the op list is normalised into dense,
// permutation and diagonal gates, a commutation-aware dependency DAG is built,
// and gates are packed greedily into tile sweeps: each sweep streams every
// amplitude through shared memory / registers once and applies every gate whose
// dense qubits lie in the sweep's tile, in an order that respects the DAG.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "sc_internal.h"

namespace sc {

static inline bool czero(double re, double im) { return re == 0.0 && im == 0.0; }

double gate_cost(const PGate& g) {
  switch (g.kind) {
    case PK_DENSE1:
    case PK_TMAT: return 8.0;     // 2 complex MACs per amplitude
    case PK_DENSE2: return 16.0;  // 4 complex MACs per amplitude
    case PK_DIAG1:
    case PK_DIAG2: return 3.0;    // 1 complex multiply + bit tests
    case PK_PAULI: return 1.0;    // a register select / sign per trajectory
    case PK_PROBE: return 2.0;    // one complex product per amplitude, reduced
    default: return 0.5;          // register selects
  }
}

int gate_pool_size(const PGate& g) {
  switch (g.kind) {
    case PK_DENSE1: return 16;  // 8 as a matrix; up to 16 in a rotation-form record
    case PK_DENSE2: return 32;
    case PK_DIAG1: return 4;
    case PK_DIAG2: return 8;
    case PK_PAULI: return 9;    // conjugated through folded permutations: (u, w, p) x 3
    default: return 0;
  }
}

uint64_t dense_mask(const PGate& g) {
  switch (g.kind) {
    case PK_DENSE1:
    case PK_PAULI:
    case PK_PROBE:
    case PK_TMAT:
    case PK_X: return 1ULL << g.q0;
    case PK_DENSE2:
    case PK_SWAP: return (1ULL << g.q0) | (1ULL << g.q1);
    default: return 0;
  }
}

uint64_t touch_mask(const PGate& g) {
  if (g.kind == PK_PAULI || g.kind == PK_TMAT) return 1ULL << g.q0;
  uint64_t m = g.cmask | (1ULL << g.q0);
  if (g.kind == PK_DENSE2 || g.kind == PK_SWAP || g.kind == PK_DIAG2) m |= 1ULL << g.q1;
  return m;
}

static void rotation(int kind, double a, double* g) {
  const double half = a / 2.0;
  const double c = std::cos(half), s = std::sin(half);
  std::memset(g, 0, 8 * sizeof(double));
  if (kind == SC_OP_RX) {
    g[0] = c; g[3] = -s; g[5] = -s; g[6] = c;
  } else {  // RY
    g[0] = c; g[2] = -s; g[4] = s; g[6] = c;
  }
}

bool normalise_op(const sc_op& op, const double* params, int64_t n_params, PGate* out,
                  bool* produced) {
  *produced = false;
  PGate g;
  std::memset(&g, 0, sizeof g);
  g.q1 = -1;
  auto angle = [&]() {
    return (op.param >= 0 && params && op.param < n_params) ? params[op.param] : op.m[0];
  };
  switch (op.kind) {
    case SC_OP_MEASURE: return true;
    case SC_OP_SINGLE:
    case SC_OP_MULTI: {
      const double* m = op.m;
      g.q0 = op.q0;
      g.cmask = (op.kind == SC_OP_MULTI) ? op.mask : 0;
      const bool off_zero = czero(m[2], m[3]) && czero(m[4], m[5]);
      const bool diag_zero = czero(m[0], m[1]) && czero(m[6], m[7]);
      if (off_zero) {
        g.kind = PK_DIAG1;
        g.m[0] = m[0]; g.m[1] = m[1]; g.m[2] = m[6]; g.m[3] = m[7];
      } else if (diag_zero && m[2] == 1.0 && m[3] == 0.0 && m[4] == 1.0 && m[5] == 0.0) {
        g.kind = PK_X;
      } else {
        g.kind = PK_DENSE1;
        std::memcpy(g.m, m, 8 * sizeof(double));
      }
      break;
    }
    case SC_OP_CNOT:
      g.kind = PK_X;
      g.q0 = op.q1;
      g.cmask = 1ULL << op.q0;
      break;
    case SC_OP_TWO: {
      g.q0 = op.q0;
      g.q1 = op.q1;
      bool diagonal = true;
      for (int r = 0; r < 4 && diagonal; ++r)
        for (int c = 0; c < 4; ++c)
          if (r != c && !czero(op.m[2 * (4 * r + c)], op.m[2 * (4 * r + c) + 1])) {
            diagonal = false;
            break;
          }
      if (diagonal) {
        g.kind = PK_DIAG2;
        for (int k = 0; k < 4; ++k) {
          g.m[2 * k] = op.m[2 * (5 * k)];
          g.m[2 * k + 1] = op.m[2 * (5 * k) + 1];
        }
      } else {
        g.kind = PK_DENSE2;
        std::memcpy(g.m, op.m, 32 * sizeof(double));
      }
      break;
    }
    case SC_OP_DIAG2:
      g.kind = PK_DIAG2;
      g.q0 = op.q0;
      g.q1 = op.q1;
      std::memcpy(g.m, op.m, 8 * sizeof(double));
      break;
    case SC_OP_SWAP:
      g.kind = PK_SWAP;
      g.q0 = op.q0;
      g.q1 = op.q1;
      break;
    case SC_OP_RX:
    case SC_OP_RY:
      g.kind = PK_DENSE1;
      g.q0 = op.q0;
      rotation(op.kind, angle(), g.m);
      break;
    case SC_OP_RZ: {
      const double h = angle() / 2.0;
      g.kind = PK_DIAG1;
      g.q0 = op.q0;
      g.m[0] = std::cos(-h); g.m[1] = std::sin(-h);
      g.m[2] = std::cos(h); g.m[3] = std::sin(h);
      break;
    }
    case SC_OP_RZZ: {
      const double h = angle() / 2.0;
      g.kind = PK_DIAG2;
      g.q0 = op.q0;
      g.q1 = op.q1;
      const double cr = std::cos(-h), ci = std::sin(-h), pr = std::cos(h), pi = std::sin(h);
      g.m[0] = cr; g.m[1] = ci; g.m[2] = pr; g.m[3] = pi;
      g.m[4] = pr; g.m[5] = pi; g.m[6] = cr; g.m[7] = ci;
      break;
    }
    default: return false;
  }
  *produced = true;
  *out = g;
  return true;
}

// ---------------------------------------------------------------------------
// planner
// ---------------------------------------------------------------------------
namespace {

struct Dag {
  std::vector<int32_t> dep_off;  // CSR
  std::vector<int32_t> deps;
};

Dag build_dag(const std::vector<PGate>& gates, int n) {
  const int G = (int)gates.size();
  Dag d;
  d.dep_off.assign(G + 1, 0);
  std::vector<int32_t> last_dense(n, -1);
  std::vector<std::vector<int32_t>> diag_since(n);
  std::vector<int32_t> tmp;
  for (int g = 0; g < G; ++g) {
    const uint64_t dm = dense_mask(gates[g]);
    const uint64_t dg = touch_mask(gates[g]) & ~dm;
    tmp.clear();
    for (uint64_t m = dm; m; m &= m - 1) {
      const int q = __builtin_ctzll(m);
      if (last_dense[q] >= 0) tmp.push_back(last_dense[q]);
      tmp.insert(tmp.end(), diag_since[q].begin(), diag_since[q].end());
    }
    for (uint64_t m = dg; m; m &= m - 1) {
      const int q = __builtin_ctzll(m);
      if (last_dense[q] >= 0) tmp.push_back(last_dense[q]);
    }
    for (uint64_t m = dm; m; m &= m - 1) {
      const int q = __builtin_ctzll(m);
      last_dense[q] = g;
      diag_since[q].clear();
    }
    for (uint64_t m = dg; m; m &= m - 1) diag_since[__builtin_ctzll(m)].push_back(g);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    d.deps.insert(d.deps.end(), tmp.begin(), tmp.end());
    d.dep_off[g + 1] = (int32_t)d.deps.size();
  }
  return d;
}

inline int popc(uint64_t x) { return __builtin_popcountll(x); }

// diag(d0, d1, d1, d0): depends only on the parity of the two bits
bool is_parity_diag(const PGate& g) {
  return g.m[0] == g.m[6] && g.m[1] == g.m[7] && g.m[2] == g.m[4] && g.m[3] == g.m[5];
}

// A 2x2 unitary u as e^{ig} c diag(1, e^{i phi}) [[1, -t], [t, 1]] diag(1, e^{i lam})
// with c = |u00| >= min_c, s = |u10| > 0, t = s / c (u00 = e^{ig} c,
// u01 = -e^{ig} e^{i lam} s, u10 = e^{ig} e^{i phi} s, u11 = e^{ig} e^{i(phi+lam)} c).
// q = {t, Re e^{i lam}, Im e^{i lam}, Re e^{i phi}, Im e^{i phi}}; (fr, fi) = e^{ig} c.
// False when u is not of that form (not unitary to 1e-13, c too small, s = 0).
bool rotation_form(const double* u, double min_c, double* q, double* fr, double* fi) {
  const double c = std::hypot(u[0], u[1]), s = std::hypot(u[4], u[5]);
  if (!(min_c > 0.0) || !(c >= min_c) || !(s > 0.0)) return false;
  if (std::fabs(c * c + s * s - 1.0) > 1e-13 || std::fabs(std::hypot(u[2], u[3]) - s) > 1e-13 ||
      std::fabs(std::hypot(u[6], u[7]) - c) > 1e-13)
    return false;
  const double gr = u[0] / c, gi = u[1] / c;  // e^{ig}
  // e^{i phi} = u10 conj(e^{ig}) / s, e^{i lam} = -u01 conj(e^{ig}) / s
  const double pr = (u[4] * gr + u[5] * gi) / s, pi = (u[5] * gr - u[4] * gi) / s;
  const double lr = -(u[2] * gr + u[3] * gi) / s, li = -(u[3] * gr - u[2] * gi) / s;
  // u11 must equal e^{ig} e^{i phi} e^{i lam} c
  const double plr = pr * lr - pi * li, pli = pr * li + pi * lr;
  const double er = c * (gr * plr - gi * pli), ei = c * (gr * pli + gi * plr);
  if (std::fabs(er - u[6]) > 1e-13 || std::fabs(ei - u[7]) > 1e-13) return false;
  q[0] = s / c;
  q[1] = lr;
  q[2] = li;
  q[3] = pr;
  q[4] = pi;
  *fr = gr * c;
  *fi = gi * c;
  return true;
}

// A 2x2 unitary u that is e^{ig} [[cos al, -sin al], [sin al, cos al]] (a real
// rotation up to a phase): the lifting shears of al reduced to |al| <= pi/2 (the
// reduction by pi is a sign, itself a phase): q = {-tan(al/2), sin al}.
bool lifted_rotation(const double* u, double* q) {
  constexpr double kTol = 1e-13;
  if (std::hypot(u[0] - u[6], u[1] - u[7]) > kTol || std::hypot(u[2] + u[4], u[3] + u[5]) > kTol)
    return false;
  const double c0 = std::hypot(u[0], u[1]), s0 = std::hypot(u[4], u[5]);
  if (std::fabs(c0 * c0 + s0 * s0 - 1.0) > kTol) return false;
  // the common phase, from the larger of u00 and u10
  const double gr = c0 >= s0 ? u[0] / c0 : u[4] / s0, gi = c0 >= s0 ? u[1] / c0 : u[5] / s0;
  // u00 e^{-ig} and u10 e^{-ig} must be real
  const double cr = u[0] * gr + u[1] * gi, ci = u[1] * gr - u[0] * gi;
  const double sr = u[4] * gr + u[5] * gi, si = u[5] * gr - u[4] * gi;
  if (std::fabs(ci) > kTol || std::fabs(si) > kTol) return false;
  double al = std::atan2(sr, cr);
  if (al > 0.5 * M_PI) al -= M_PI;
  if (al < -0.5 * M_PI) al += M_PI;
  q[0] = -std::tan(0.5 * al);
  q[1] = std::sin(al);
  return true;
}

// ---------------------------------------------------------------------------
// Stage peephole: fewer records per stage.  Every record costs a dispatch and a
// reconciliation of the register-resident amplitudes, so register-bit diagonals
// are moved towards the start of the stage (conjugated through plain register
// permutations: d'(x) = d(P x) for an involution P), merged into the phase table of
// a rotation-form record that covers their bits, and plain permutations that end
// up last to touch their bits are folded into the stage's exit permutation.
// ---------------------------------------------------------------------------
namespace {

bool sk_diagonal(int32_t k) {
  return k == SK_D1 || k == SK_D2 || k == SK_DP || k == SK_D1R || k == SK_DPR;
}

// register bits a record reads or writes (tile positions mapped through reg_of_pos)
uint32_t record_bits(const SwGate& g, const int* reg_of_pos) {
  uint32_t f = 0;
  auto reg = [&](int p) {
    if (p >= 0 && p < 32 && reg_of_pos[p] >= 0) f |= 1u << reg_of_pos[p];
  };
  switch (g.kind) {
    case SK_G1: case SK_X: case SK_X0: case SK_D1R: case SK_PAULI: case SK_XF: case SK_TMAT:
    case SK_D1H:
      f |= 1u << g.a;
      break;
    case SK_G2: case SK_CX: case SK_CX0: case SK_DPR: case SK_SWAP: case SK_CXF:
      f |= (1u << g.a) | (1u << g.b);
      break;
    case SK_G1ALL: case SK_G1ALLQ: case SK_ROTL: f |= (uint32_t)g.a & 15u; break;
    case SK_DTAB: f |= 15u; break;
    case SK_D1: reg(g.a); break;
    case SK_DP: case SK_D2: reg(g.a); reg(g.b); break;
    default: return 0xFFFFFFFFu;
  }
  for (uint32_t m = g.lmask; m; m &= m - 1) reg(__builtin_ctz(m));
  return f;
}

// X / CX / SWAP on register bits with no tile or global controls
bool plain_permutation(const SwGate& g) {
  return (g.kind == SK_X0 || g.kind == SK_CX0 || g.kind == SK_SWAP) && g.gmask == 0 && g.lmask == 0;
}

// register bits a plain permutation changes (a SWAP's both, an X's target)
uint32_t written_bits(const SwGate& p) {
  return p.kind == SK_SWAP ? (1u << p.a) | (1u << p.b) : 1u << p.a;
}

// X / CX on register bits whose other controls lie outside the registers
bool conditional_permutation(const SwGate& g, const int* reg_of_pos) {
  if (g.kind == SK_X0 || g.kind == SK_X) return record_bits(g, reg_of_pos) == 1u << g.a;
  if (g.kind == SK_CX0 || g.kind == SK_CX)
    return record_bits(g, reg_of_pos) == ((1u << g.a) | (1u << g.b));
  return false;
}

bool register_diagonal(const SwGate& g) {
  return (g.kind == SK_D1R || g.kind == SK_DPR) && g.gmask == 0 && g.lmask == 0;
}

// entry of a D1R / DPR record (pool: two complex values) at register index x
void diagonal_at(const SwGate& d, const std::vector<double>& pool, int x, double* re, double* im) {
  const int k = d.kind == SK_D1R ? (x >> d.a) & 1 : ((x >> d.a) ^ (x >> d.b)) & 1;
  *re = pool[d.moff + 2 * k];
  *im = pool[d.moff + 2 * k + 1];
}

// Rewrites diagonal d (applied after plain permutation p) as the diagonal to apply
// before p; false when the result is not a D1R / DPR record.
bool conjugate_diagonal(SwGate& d, const SwGate& p, std::vector<double>& pool) {
  const uint32_t db = d.kind == SK_D1R ? 1u << d.a : (1u << d.a) | (1u << d.b);
  auto set = [&](int32_t kind, int32_t a, int32_t b) {
    d.kind = kind;
    d.a = a;
    d.b = b;
    d.code = sw_code(kind, a, b);
  };
  if (p.kind == SK_X0) {  // d(x ^ e_a): the entries trade places when a is one of d's bits
    if ((db >> p.a) & 1) {
      std::swap(pool[d.moff], pool[d.moff + 2]);
      std::swap(pool[d.moff + 1], pool[d.moff + 3]);
    }
    return true;
  }
  if (p.kind == SK_SWAP) {
    auto map = [&](int32_t b) { return b == p.a ? p.b : (b == p.b ? p.a : b); };
    if (d.kind == SK_D1R) set(SK_D1R, map(d.a), 0);
    else set(SK_DPR, map(d.a), map(d.b));
    return true;
  }
  if (p.kind == SK_CX0) {  // target p.a, control p.b: x_t -> x_t ^ x_c
    const int32_t t = p.a, c = p.b;
    if (!((db >> t) & 1)) return true;
    if (d.kind == SK_D1R) {  // d(x_t ^ x_c): a parity diagonal on (t, c)
      set(SK_DPR, t, c);
      return true;
    }
    const int32_t o = d.a == t ? d.b : d.a;
    if (o == c) {  // parity of (x_t ^ x_c, x_c) is x_t
      set(SK_D1R, t, 0);
      return true;
    }
  }
  return false;
}

// Merges unitary diagonal d into the output (after) or input (before) phase table of
// rotation-form record g when d's bits are among g's; d(0) joins the sweep scalar.
bool merge_diagonal(const SwGate& g, const SwGate& d, bool after, std::vector<double>& pool,
                    double* sr, double* si) {
  const uint32_t M = (uint32_t)g.a & 15u;
  const uint32_t db = d.kind == SK_D1R ? 1u << d.a : (1u << d.a) | (1u << d.b);
  if (g.kind != SK_G1ALLQ || g.gmask || g.lmask || (db & ~M)) return false;
  int bits[4], K = 0;
  for (int b = 0; b < 4; ++b)
    if ((M >> b) & 1) bits[K++] = b;
  double e[4];
  for (int k = 0; k < 2; ++k) {
    e[2 * k] = pool[d.moff + 2 * k];
    e[2 * k + 1] = pool[d.moff + 2 * k + 1];
    if (std::fabs(e[2 * k] * e[2 * k] + e[2 * k + 1] * e[2 * k + 1] - 1.0) > 1e-12) return false;
  }
  double d0r, d0i;
  diagonal_at(d, pool, 0, &d0r, &d0i);
  const int base = g.moff + 2 * K + (after ? 2 * ((1 << K) - 1) : 0);
  for (int s = 1; s < (1 << K); ++s) {
    int x = 0;
    for (int k = 0; k < K; ++k)
      if ((s >> k) & 1) x |= 1 << bits[k];
    double dr, di;
    diagonal_at(d, pool, x, &dr, &di);
    const double rr = dr * d0r + di * d0i, ri = di * d0r - dr * d0i;  // d(x) / d(0)
    double& tr = pool[base + 2 * (s - 1)];
    double& ti = pool[base + 2 * (s - 1) + 1];
    const double nr = tr * rr - ti * ri, ni = tr * ri + ti * rr;
    tr = nr;
    ti = ni;
  }
  const double nr = *sr * d0r - *si * d0i, ni = *sr * d0i + *si * d0r;
  *sr = nr;
  *si = ni;
  return true;
}

// exit permutation of a stage after plain permutation p (applied at the end)
void compose_permutation(SwStage& st, const SwGate& p) {
  for (int j = 0; j < 16; ++j) {
    int x = st.perm[j];
    if (p.kind == SK_SWAP) {
      if (((x >> p.a) ^ (x >> p.b)) & 1) x ^= (1 << p.a) | (1 << p.b);
    } else if (p.kind == SK_X0) {
      x ^= 1 << p.a;
    } else if ((x >> p.b) & 1) {
      x ^= 1 << p.a;
    }
    st.perm[j] = (int8_t)x;
  }
}

// folded_bits: register bits of the permutations folded while the stage was built;
// last: the sweep's last stage (its exit is the global store: no slot folds)
void optimize_stage(Plan& plan, int32_t g0, SwStage& st, const int* reg_of_pos,
                    uint32_t folded_bits, bool last, double* sr, double* si) {
  std::vector<SwGate>& G = plan.gates;
  for (int i = g0; i < (int)G.size(); ++i) {
    if (!sk_diagonal(G[i].kind)) continue;
    const bool reg_diag = register_diagonal(G[i]);
    int j = i;
    bool merged = false;
    while (j > g0) {
      const SwGate& p = G[j - 1];
      if (reg_diag && merge_diagonal(p, G[j], true, plan.pool, sr, si)) {
        merged = true;
        break;
      }
      const uint32_t df = record_bits(G[j], reg_of_pos);
      if (sk_diagonal(p.kind) || !(record_bits(p, reg_of_pos) & df) ||
          (plain_permutation(p) && !(written_bits(p) & df))) {
        std::swap(G[j - 1], G[j]);
        --j;
        continue;
      }
      if (reg_diag && plain_permutation(p)) {
        SwGate d = G[j];
        if (conjugate_diagonal(d, p, plan.pool)) {
          G[j] = p;
          G[j - 1] = d;
          --j;
          continue;
        }
      }
      break;
    }
    if (merged) {
      G.erase(G.begin() + j);
      --i;
    }
  }
  // Folds, decided backwards.  A plain permutation folds when no later record other
  // than a Pauli slot touches its bits: the slots after it are conjugated below, and
  // folded permutations may overlap (they compose in time order).  Slot folds of
  // conditional permutations need every later record, slots included, off their bits.
  const int ng = (int)G.size() - g0;
  std::vector<char> fold(ng, 0);
  uint32_t later_all = folded_bits, later = folded_bits;
  for (int k = (int)G.size() - 1; k >= g0; --k) {
    SwGate& g = G[k];
    const uint32_t f = record_bits(g, reg_of_pos);
    if (plain_permutation(g) && !(f & later)) {
      fold[k - g0] = 1;
      later_all |= f;
      continue;
    }
    if (!last && !(f & later_all) && conditional_permutation(g, reg_of_pos)) {
      g.kind = (g.kind == SK_X0 || g.kind == SK_X) ? SK_XF : SK_CXF;
      g.code = sw_code(g.kind, g.a, g.b);
    }
    later_all |= f;
    if (g.kind != SK_PAULI) later |= f;
  }
  // Forwards: the folded permutations join the exit permutation in time order; a
  // slot after some of them becomes P^dag S P, P their composition (x -> M x ^ c):
  // X_a -> X^{M^-1 e_a}, Z_a -> (-1)^{c_a} Z^{M^T e_a}, Y_a = i X_a Z_a likewise.
  SwStage pst;
  for (int j = 0; j < 16; ++j) pst.perm[j] = (int8_t)j;
  bool moved = false;
  for (int k = g0; k < (int)G.size(); ++k) {
    SwGate& g = G[k];
    if (fold[k - g0]) {
      compose_permutation(st, g);
      compose_permutation(pst, g);
      moved = true;
      continue;
    }
    if (g.kind != SK_PAULI || !moved) continue;
    const int a = g.a, c = pst.perm[0];
    int u = 0, w = 0;
    for (int x = 0; x < 16; ++x)
      if ((pst.perm[x] ^ c) == (1 << a)) u = x;  // M^-1 e_a
    for (int b = 0; b < 4; ++b) w |= (((pst.perm[1 << b] ^ c) >> a) & 1) << b;  // M^T e_a
    const int sa = (c >> a) & 1;
    if (u == (1 << a) && w == (1 << a) && sa == 0) continue;  // P commutes with the slot
    g.kind = SK_PAULIF;
    g.moff = (int32_t)plan.pool.size();
    g.code = SK_PAULIF << 4;
    const double frame[9] = {(double)u, 0.0, 0.0,                      // X
                             (double)u, (double)w, (double)(1 + 2 * sa),  // Y = i X Z
                             0.0, (double)w, (double)(2 * sa)};        // Z
    plan.pool.insert(plan.pool.end(), frame, frame + 9);
  }
  for (int k = (int)G.size() - 1; k >= g0; --k)
    if (fold[k - g0]) G.erase(G.begin() + k);
}

// Runs of two or more adjacent register-bit diagonals (D1R / DPR without tile or
// global controls) become one SK_DTAB record: their product as a table over the
// stage's 2^nr register indices.  They commute, so the order inside a run is free.
// pool_limit: the end of the sweep's pool budget (a table that would pass it is not
// made).
void merge_register_diagonals(Plan& plan, int32_t g0, int nr, size_t pool_limit) {
  std::vector<SwGate>& G = plan.gates;
  for (int i = g0; i < (int)G.size(); ++i) {
    if (!register_diagonal(G[i])) continue;
    int j = i;
    while (j + 1 < (int)G.size() && register_diagonal(G[j + 1])) ++j;
    if (j == i) continue;
    if (plan.pool.size() + (2u << nr) > pool_limit) return;
    SwGate t;
    std::memset(&t, 0, sizeof t);
    t.kind = SK_DTAB;
    t.code = sw_code(SK_DTAB, 0, 0);
    t.moff = (int32_t)plan.pool.size();
    std::vector<double> tab(2 * ((size_t)1 << nr));
    for (int x = 0; x < (1 << nr); ++x) {
      double pr = 1.0, pi = 0.0;
      for (int k = i; k <= j; ++k) {
        double dr, di;
        diagonal_at(G[k], plan.pool, x, &dr, &di);
        const double nr_ = pr * dr - pi * di, ni = pr * di + pi * dr;
        pr = nr_;
        pi = ni;
      }
      tab[2 * x] = pr;
      tab[2 * x + 1] = pi;
    }
    plan.pool.insert(plan.pool.end(), tab.begin(), tab.end());
    G.erase(G.begin() + i + 1, G.begin() + j + 1);
    G[i] = t;
  }
}

}  // namespace

// In-place bit permutations that take the layout phys_of back to the identity:
// transpositions of physical bits, grouped while their bits (plus the low bits,
// which keep the copies coalesced) fit one permutation tile.
std::vector<SwPerm> restore_identity(const int* phys_in, int n) {
  int phys_of[64], log_of[64];
  for (int q = 0; q < n; ++q) {
    phys_of[q] = phys_in[q];
    log_of[phys_in[q]] = q;
  }
  std::vector<std::pair<int, int>> swaps;
  for (int q = 0; q < n; ++q) {
    const int b = phys_of[q];
    if (b == q) continue;
    const int r = log_of[q];  // the qubit on bit q moves to bit b
    swaps.emplace_back(q, b);
    phys_of[q] = q; log_of[q] = q;
    phys_of[r] = b; log_of[b] = r;
  }
  std::vector<SwPerm> out;
  const int base_bits = std::min(n, 4);
  size_t i = 0;
  while (i < swaps.size()) {
    uint64_t S = (base_bits >= 64) ? ~0ULL : ((1ULL << base_bits) - 1ULL);
    int cur[64];
    for (int b = 0; b < 64; ++b) cur[b] = b;
    size_t j = i;
    for (; j < swaps.size(); ++j) {
      const uint64_t S2 = S | (1ULL << swaps[j].first) | (1ULL << swaps[j].second);
      if (popc(S2) > SW_PERM_MAX_BITS) break;
      S = S2;
      std::swap(cur[swaps[j].first], cur[swaps[j].second]);
    }
    SwPerm pm;
    std::memset(&pm, 0, sizeof pm);
    int idx[64];
    for (uint64_t m = S; m; m &= m - 1) {
      const int b = __builtin_ctzll(m);
      idx[b] = pm.nbits;
      pm.bits[pm.nbits++] = (int8_t)b;
    }
    for (int k = 0; k < pm.nbits; ++k) pm.src[k] = (int8_t)idx[cur[pm.bits[k]]];
    out.push_back(pm);
    i = j;
  }
  return out;
}

}  // namespace

// Entry folds (StageEntry): the records that open stage st and only permute its
// registers are taken out of its range and composed into the read.  Record i acts as
// new v[j] = old v[pi_i(j)]; after the prefix, v[j] = read[sigma(j)] with
// sigma = pi_1 o pi_2 o ...  A conditional X on register bit a (controls outside the
// registers) translates by e_a where its condition holds, which moves sigma's
// result by the linear part of the composition so far applied to e_a (rf_d).
void fold_stage_entry(const Plan& plan, SwStage& st, StageEntry* en) {
  const int nv = 1 << st.nr;
  uint32_t regpos = 0;
  for (int k = 0; k < st.nr; ++k) regpos |= 1u << st.R[k];
  int sigma[16];
  for (int j = 0; j < 16; ++j) sigma[j] = j;
  int g = st.g0;
  for (; g < st.g1; ++g) {
    const SwGate& q = plan.gates[g];
    int pi[16];
    for (int j = 0; j < 16; ++j) pi[j] = j;
    const bool plain = q.lmask == 0 && q.gmask == 0;
    if (plain && q.kind == SK_X0) {
      for (int j = 0; j < nv; ++j) pi[j] = j ^ (1 << q.a);
    } else if (plain && q.kind == SK_CX0) {
      for (int j = 0; j < nv; ++j) pi[j] = ((j >> q.b) & 1) ? j ^ (1 << q.a) : j;
    } else if (plain && q.kind == SK_SWAP) {
      for (int j = 0; j < nv; ++j) {
        const int ba = (j >> q.a) & 1, bb = (j >> q.b) & 1;
        pi[j] = ba == bb ? j : j ^ ((1 << q.a) | (1 << q.b));
      }
    } else if ((q.kind == SK_X0 || q.kind == SK_X) && !(q.lmask & regpos) &&
               en->n_rf < kEntryMaxCond) {
      // the translation's delta through the linear part of sigma
      en->rf_g[en->n_rf] = g;
      en->rf_d[en->n_rf] = sigma[1 << q.a] ^ sigma[0];
      ++en->n_rf;
      continue;
    } else {
      break;
    }
    int nsig[16];
    for (int j = 0; j < 16; ++j) nsig[j] = j < nv ? sigma[pi[j]] : j;
    for (int j = 0; j < 16; ++j) sigma[j] = nsig[j];
  }
  for (int j = 0; j < 16; ++j) en->rperm[j] = (int8_t)sigma[j];
  st.g0 = g;
}

Plan plan_sweeps(const std::vector<PGate>& gates, int n, const PlanParams& pp) {
  Plan plan;
  const int G = (int)gates.size();
  plan.n_gates = G;
  if (G == 0) return plan;

  // a stage must hold both qubits of a two-qubit gate
  const int NR = std::min(std::max(pp.nr, 2), n);
  const int L0 = std::min(pp.low_qubits, n);
  int T = std::min(pp.tile_qubits, n);
  // keep at least 2^8 tiles per sweep when the state allows it
  if (n - T < 8) T = n - 8;
  // the tile must hold a stage's registers and two high qubits (a 2-qubit gate)
  T = std::max(T, std::min(n, std::max(NR, L0 + 2)));
  const int L = std::min(L0, T);
  const int h = T - L;
  const bool high_edges = h >= NR;  // first/last stage can use only high positions
  // qubit layout (logical <-> physical), identity at the start and the end
  int phys_of[64], log_of[64];
  for (int q = 0; q < 64; ++q) phys_of[q] = log_of[q] = q;
  const bool use_relayout = pp.relayout && high_edges && L >= 1 && n > T;
  // unscheduled gates the relayout lookahead inspects
  const int kLookahead = 8 * T;
  constexpr int kNever = 1 << 30;

  Dag dag = build_dag(gates, n);
  std::vector<int32_t> when(G, -1);
  std::vector<int32_t> idx_in_sweep(G, -1);
  int first = 0;
  int sweep_id = 0;
  std::vector<int32_t> list;
  std::vector<char> staged;

  while (first < G) {
    // logical qubits on the contiguous low physical bits: free for this sweep
    uint64_t low_qmask = 0;
    for (int p = 0; p < L; ++p) low_qmask |= 1ULL << log_of[p];
    uint64_t H = 0;
    int hcount = 0;
    double used = 0.0;
    int pool_used = 0;
    list.clear();
    for (int g = first; g < G; ++g) {
      if (when[g] >= 0) continue;
      bool ok = true;
      for (int k = dag.dep_off[g]; k < dag.dep_off[g + 1]; ++k)
        if (when[dag.deps[k]] < 0) { ok = false; break; }
      if (!ok) continue;
      const uint64_t need = dense_mask(gates[g]) & ~low_qmask & ~H;
      const int c = popc(need);
      if (hcount + c > h) continue;
      const double cost = gate_cost(gates[g]);
      if (pp.budget >= 0 && !list.empty() && used + cost > pp.budget) break;
      if ((int)list.size() >= pp.max_gates) break;
      if (pool_used + gate_pool_size(gates[g]) > pp.max_pool) break;
      H |= need;
      hcount += c;
      used += cost;
      pool_used += gate_pool_size(gates[g]);
      when[g] = sweep_id;
      list.push_back(g);
    }
    // lookahead: rank of the first later gate that needs each qubit in a tile
    int first_need[64];
    for (int q = 0; q < 64; ++q) first_need[q] = kNever;
    bool more = false;
    {
      int seen = 0;
      for (int g = first; g < G && seen < kLookahead; ++g) {
        if (when[g] >= 0) continue;
        more = true;
        ++seen;
        for (uint64_t m = dense_mask(gates[g]); m; m &= m - 1) {
          const int q = __builtin_ctzll(m);
          if (first_need[q] == kNever) first_need[q] = seen;
        }
      }
      for (int g = first; g < G && !more; ++g) more = when[g] < 0;
    }
    // pad the high set to exactly h qubits so every sweep tile has 2^T amplitudes;
    // qubits needed soonest first, so a relayout can bring them low
    if (hcount < h) {
      std::vector<int> cand;
      for (int q = 0; q < n; ++q)
        if (!((low_qmask >> q) & 1ULL) && !((H >> q) & 1ULL)) cand.push_back(q);
      // ties: qubits away from their home bit first (a chance to send them home)
      std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) {
        if (first_need[a] != first_need[b]) return first_need[a] < first_need[b];
        const bool ma = phys_of[a] != a, mb = phys_of[b] != b;
        if (ma != mb) return ma;
        return phys_of[a] < phys_of[b];
      });
      for (size_t k = 0; k < cand.size() && hcount < h; ++k) {
        H |= 1ULL << cand[k];
        ++hcount;
      }
    }

    // relayout: swap up to NR high qubits needed soon with low qubits needed later
    // (after the last gates: the qubits whose home is low come back)
    std::vector<int> incoming, outgoing;
    if (use_relayout) {
      auto need_rank = [&](int q) {
        if (more) return first_need[q];
        return q < L ? 0 : kNever;
      };
      std::vector<int> in_c, out_c;
      for (uint64_t m = H; m; m &= m - 1) in_c.push_back(__builtin_ctzll(m));
      for (int p = 0; p < L; ++p) out_c.push_back(log_of[p]);
      std::stable_sort(in_c.begin(), in_c.end(),
                       [&](int a, int b) { return need_rank(a) < need_rank(b); });
      std::stable_sort(out_c.begin(), out_c.end(),
                       [&](int a, int b) { return need_rank(a) > need_rank(b); });
      for (size_t k = 0; k < in_c.size() && k < out_c.size() && (int)k < NR; ++k) {
        if (need_rank(in_c[k]) >= need_rank(out_c[k])) break;
        incoming.push_back(in_c[k]);
        outgoing.push_back(out_c[k]);
      }
    }
    const int n_in = (int)incoming.size();

    SwSweep sw;
    std::memset(&sw, 0, sizeof sw);
    sw.T = T; sw.L = L; sw.h = h; sw.nr = NR;
    sw.scale_re = 1.0;
    sw.scale_im = 0.0;
    sw.tiles = 1LL << (n - T);
    int pos_of[64];
    int log_at[32];  // logical qubit at each tile position
    for (int q = 0; q < 64; ++q) pos_of[q] = -1;
    for (int p = 0; p < L; ++p) {
      pos_of[log_of[p]] = p;
      log_at[p] = log_of[p];
    }
    {
      // incoming qubits take the first high positions, the rest follow by physical bit
      std::vector<int> order(incoming.begin(), incoming.end());
      std::sort(order.begin(), order.end(),
                [&](int a, int b) { return phys_of[a] < phys_of[b]; });
      std::vector<int> rest;
      for (uint64_t m = H; m; m &= m - 1) {
        const int q = __builtin_ctzll(m);
        if (std::find(incoming.begin(), incoming.end(), q) == incoming.end()) rest.push_back(q);
      }
      std::sort(rest.begin(), rest.end(), [&](int a, int b) { return phys_of[a] < phys_of[b]; });
      order.insert(order.end(), rest.begin(), rest.end());
      for (int k = 0; k < h; ++k) {
        sw.hq[k] = phys_of[order[k]];
        sw.hs[k] = sw.hq[k];
        pos_of[order[k]] = L + k;
        log_at[L + k] = order[k];
      }
      std::sort(sw.hs, sw.hs + h);
    }
    // output layout: staying low qubits, then incoming ones, on the low physical bits;
    // every other tile qubit goes to its home bit when that bit is in the tile
    uint32_t out_pos = 0;  // positions of the outgoing qubits
    for (int q : outgoing) out_pos |= 1u << pos_of[q];
    {
      int next_low = 0;
      for (int p = 0; p < L; ++p)
        if (!((out_pos >> p) & 1u)) sw.outp[p] = (int8_t)next_low++;
      for (int k = 0; k < n_in; ++k) sw.outp[L + k] = (int8_t)next_low++;
      std::vector<char> taken(64, 0);
      std::vector<int> rest_pos;
      for (int p = 0; p < T; ++p) {
        const bool low_dest = (p < L && !((out_pos >> p) & 1u)) || (p >= L && p < L + n_in);
        if (!low_dest) rest_pos.push_back(p);
      }
      // the low bits all went to staying / incoming qubits: the rest share the high bits
      std::vector<int> avail(sw.hq, sw.hq + h);
      std::vector<char> done(32, 0);
      for (int p : rest_pos) {
        const int home = log_at[p];
        if (home >= L && std::find(avail.begin(), avail.end(), home) != avail.end() && !taken[home]) {
          sw.outp[p] = (int8_t)home;
          taken[home] = 1;
          done[p] = 1;
        }
      }
      std::sort(avail.begin(), avail.end());
      size_t ai = 0;
      for (int p : rest_pos) {
        if (done[p]) continue;
        while (taken[avail[ai]]) ++ai;
        sw.outp[p] = (int8_t)avail[ai];
        taken[avail[ai]] = 1;
      }
    }
    for (int p = 0; p < T; ++p) {
      const int in_phys = p < L ? p : sw.hq[p - L];
      if (sw.outp[p] != in_phys) sw.relayout = 1;
    }
    const uint32_t high_pos = (T >= 32 ? 0xFFFFFFFFu : ((1u << T) - 1u)) & ~((1u << L) - 1u);
    const uint32_t in_pos = ((1u << n_in) - 1u) << L;  // positions of the incoming qubits
    const uint64_t tile_qmask = low_qmask | H;

    // ---- stages -----------------------------------------------------------
    for (size_t i = 0; i < list.size(); ++i) idx_in_sweep[list[i]] = (int32_t)i;
    staged.assign(list.size(), 0);
    size_t remaining = list.size();
    sw.s0 = (int32_t)plan.stages.size();
    sw.pool0 = (int32_t)plan.pool.size();
    std::vector<std::pair<uint32_t, std::vector<int32_t>>> stage_list;
    // folded[i]: list gate i is a permutation folded into its stage's exit permutation
    std::vector<char> folded(list.size(), 0);
    while (remaining > 0 || stage_list.empty()) {
      const bool first_stage = stage_list.empty();
      uint32_t R = 0;
      std::vector<int32_t> sg;
      for (size_t i = 0; i < list.size(); ++i) {
        if (staged[i]) continue;
        const int g = list[i];
        bool ok = true;
        for (int k = dag.dep_off[g]; k < dag.dep_off[g + 1]; ++k) {
          const int dpd = dag.deps[k];
          if (when[dpd] == sweep_id && !staged[idx_in_sweep[dpd]]) { ok = false; break; }
        }
        if (!ok) continue;
        uint32_t touch = 0;
        for (uint64_t m = touch_mask(gates[g]); m; m &= m - 1) {
          const int q = __builtin_ctzll(m);
          if (pos_of[q] >= 0) touch |= 1u << pos_of[q];
        }
        uint32_t need = 0;
        for (uint64_t m = dense_mask(gates[g]); m; m &= m - 1)
          need |= 1u << pos_of[__builtin_ctzll(m)];
        need &= ~R;
        if (first_stage && high_edges && (need & ~high_pos)) continue;
        if (popc(R) + popc(need) > NR) continue;
        // Positions that make the gate cheaper when they are register bits too: the
        // control of a controlled X (a register permutation) and both bits of a
        // parity diagonal (a compile-time phase pattern).  Taken only if they fit.
        uint32_t want = 0;
        const PGate& pw = gates[g];
        if (pw.kind == PK_X) {
          for (uint64_t m = pw.cmask; m; m &= m - 1) {
            const int c = __builtin_ctzll(m);
            if (pos_of[c] >= 0) {
              want |= 1u << pos_of[c];
              break;
            }
          }
        } else if (pw.kind == PK_DIAG2 && is_parity_diag(pw) && pos_of[pw.q0] >= 0 &&
                   pos_of[pw.q1] >= 0) {
          want = (1u << pos_of[pw.q0]) | (1u << pos_of[pw.q1]);
        } else if (pw.kind == PK_DIAG1 && pw.cmask == 0 && pos_of[pw.q0] >= 0) {
          want = 1u << pos_of[pw.q0];
        }
        want &= ~R & ~need;
        if (first_stage && high_edges) want &= high_pos;
        if (popc(R) + popc(need) + popc(want) <= NR) need |= want;
        R |= need;
        sg.push_back((int32_t)i);
        staged[i] = 1;
      }
      if (sg.empty() && !first_stage) {  // cannot happen for a valid DAG
        plan.ok = false;
        return plan;
      }
      // X / CNOT / SWAP acting only on register bits is a register permutation: it
      // is folded into the stage's exit permutation (no data moves) when no later
      // gate of the stage touches its bits, and executed in registers otherwise
      {
        uint32_t later = 0;
        for (size_t k = sg.size(); k-- > 0;) {
          const int32_t i = sg[k];
          const PGate& pw = gates[list[i]];
          uint32_t touch = 0;
          for (uint64_t m = touch_mask(pw); m; m &= m - 1) {
            const int q = __builtin_ctzll(m);
            if (pos_of[q] >= 0) touch |= 1u << pos_of[q];
          }
          bool fold = false;
          if (pw.kind == PK_SWAP) {
            fold = true;
          } else if (pw.kind == PK_X && (pw.cmask & ~tile_qmask) == 0 && popc(pw.cmask) <= 1) {
            fold = pw.cmask == 0 || ((touch & ~R) == 0);
          }
          if (fold && !(touch & later)) folded[i] = 1;
          later |= touch;
        }
      }
      remaining -= sg.size();
      stage_list.emplace_back(R, std::move(sg));
    }
    // The last stage's lanes must walk the positions that land on the low physical
    // bits: without a low swap those are positions 0..L-1 (registers high only);
    // with one, registers hold exactly the outgoing low positions plus high ones
    // past the incoming positions.  Otherwise a trailing empty stage does the store.
    {
      const uint32_t Rl = stage_list.back().first;
      const bool single = stage_list.size() == 1;
      bool fits;
      if (n_in == 0)
        fits = !high_edges || !(Rl & ~high_pos);
      else
        fits = !single && !(Rl & ~high_pos & ~out_pos) && !(Rl & in_pos) &&
               popc(Rl | out_pos) <= NR;
      if (!fits) stage_list.emplace_back(0u, std::vector<int32_t>());
    }

    for (size_t s = 0; s < stage_list.size(); ++s) {
      uint32_t R = stage_list[s].first;
      const bool is_last = s + 1 == stage_list.size();
      const bool edge = (s == 0) || is_last;
      if (is_last && n_in > 0) {
        R |= out_pos;
        for (int p = L + n_in; p < T && popc(R) < NR; ++p) R |= 1u << p;
      }
      // pad R to NR positions: high positions on the edges, low ones elsewhere
      if (edge && high_edges) {
        for (int p = L; p < T && popc(R) < NR; ++p) R |= 1u << p;
      }
      for (int p = 0; p < T && popc(R) < NR; ++p) R |= 1u << p;
      SwStage st;
      std::memset(&st, 0, sizeof st);
      st.nr = NR;
      int reg_of_pos[32];
      for (int p = 0; p < 32; ++p) reg_of_pos[p] = -1;
      {
        int k = 0;
        for (uint32_t m = R; m; m &= m - 1) {
          const int p = __builtin_ctz(m);
          st.R[k] = (int8_t)p;
          reg_of_pos[p] = k;
          ++k;
        }
      }
      st.g0 = (int32_t)plan.gates.size();
      for (int j = 0; j < 16; ++j) st.perm[j] = (int8_t)j;
      std::vector<int64_t> folded_ops;
      uint32_t folded_bits = 0;
      // runs of uncontrolled 2x2 gates on distinct register bits become one record
      std::vector<std::pair<int, const double*>> run;
      std::vector<int64_t> run_ops;
      // rotation-form record for the gates of `part` (increasing register bit); the
      // gates of `xpart` are U X in rotation form, so the record starts with X on them
      auto emit_rotation = [&](const std::vector<int>& part, const std::vector<double>& qs,
                               const std::vector<int>& xpart) {
        SwGate sg;
        std::memset(&sg, 0, sizeof sg);
        sg.moff = (int32_t)plan.pool.size();
        sg.kind = SK_G1ALLQ;
        for (int i : part) sg.a |= 1 << run[i].first;
        for (int i : xpart) sg.b |= 1 << run[i].first;
        // t and t / (1 + t^2) per gate, then the input- and output-phase tables over
        // the subsets s of the record's gates (bit k of s: gate k, in increasing
        // register bit).  The input table also carries the real factor 1 + t_k^2 of
        // every gate k in s: with the amplitude on the 1 side of bit k scaled by it,
        // the rotation is two in-place shears, a0 -= t/(1+t^2) a1, a1 += t a0
        // (= [[1, -t], [t, 1]] applied to the unscaled pair).
        const int K = (int)part.size();
        for (int k = 0; k < K; ++k) plan.pool.push_back(qs[5 * k]);
        for (int k = 0; k < K; ++k) plan.pool.push_back(qs[5 * k] / (1.0 + qs[5 * k] * qs[5 * k]));
        for (int side = 0; side < 2; ++side) {
          for (int sub = 1; sub < (1 << K); ++sub) {
            double pr = 1.0, pi = 0.0;
            for (int k = 0; k < K; ++k) {
              if (!((sub >> k) & 1)) continue;
              const double er = qs[5 * k + 1 + 2 * side], ei = qs[5 * k + 2 + 2 * side];
              double nr = pr * er - pi * ei, ni = pr * ei + pi * er;
              if (side == 0) {
                const double f = 1.0 + qs[5 * k] * qs[5 * k];
                nr *= f;
                ni *= f;
              }
              pr = nr;
              pi = ni;
            }
            plan.pool.push_back(pr);
            plan.pool.push_back(pi);
          }
        }
        sg.code = sw_code(sg.kind, sg.a, sg.b);
        plan.gates.push_back(sg);
        for (int i : part) plan.gate_ops.push_back(run_ops[i]);
      };
      // lifted-rotation record (phase-free plans) for the gates of `part`
      // (increasing register bit), lifting shears in `qs`
      auto emit_lifted = [&](const std::vector<int>& part, const std::vector<double>& qs) {
        SwGate sg;
        std::memset(&sg, 0, sizeof sg);
        sg.moff = (int32_t)plan.pool.size();
        sg.kind = SK_ROTL;
        for (int i : part) sg.a |= 1 << run[i].first;
        plan.pool.insert(plan.pool.end(), qs.begin(), qs.end());
        sg.code = sw_code(sg.kind, sg.a, sg.b);
        plan.gates.push_back(sg);
        for (int i : part) plan.gate_ops.push_back(run_ops[i]);
      };
      // matrix record (G1 or G1ALL) for the gates of `part` (increasing register bit)
      auto emit_matrix = [&](const std::vector<int>& part) {
        SwGate sg;
        std::memset(&sg, 0, sizeof sg);
        sg.moff = (int32_t)plan.pool.size();
        if (part.size() == 1) {
          sg.kind = SK_G1;
          sg.a = run[part[0]].first;
        } else {
          sg.kind = SK_G1ALL;
          for (int i : part) sg.a |= 1 << run[i].first;
        }
        for (int i : part) plan.pool.insert(plan.pool.end(), run[i].second, run[i].second + 8);
        sg.code = sw_code(sg.kind, sg.a, sg.b);
        plan.gates.push_back(sg);
        for (int i : part) plan.gate_ops.push_back(run_ops[i]);
      };
      // The run's gates act on distinct register bits and commute: those with a
      // rotation form make one rotation-form record, the others one matrix record.
      auto flush_run = [&]() {
        if (run.empty()) return;
        std::vector<int> order(run.size());
        for (size_t i = 0; i < run.size(); ++i) order[i] = (int)i;
        std::sort(order.begin(), order.end(), [&](int x, int y) { return run[x].first < run[y].first; });
        std::vector<int> rot, mat, xrot;
        std::vector<double> qs;
        if (pp.phase_free) {
          for (int i : order) {
            double q[2];
            if (lifted_rotation(run[i].second, q)) {
              rot.push_back(i);
              qs.insert(qs.end(), q, q + 2);
            } else {
              mat.push_back(i);
            }
          }
          if (!rot.empty()) emit_lifted(rot, qs);
          if (!mat.empty()) emit_matrix(mat);
          run.clear();
          run_ops.clear();
          return;
        }
        double sr = sw.scale_re, si = sw.scale_im;
        for (int i : order) {
          double q[5], fr, fi;
          bool ok = rotation_form(run[i].second, pp.rot_min_c, q, &fr, &fi);
          bool lead_x = false;
          if (!ok) {
            // |u00| small: U = (U X) X, and U X (the columns of U swapped) has
            // |(U X)00| = |u01| close to 1, so it takes the rotation form after an X
            const double* u = run[i].second;
            const double ux[8] = {u[2], u[3], u[0], u[1], u[6], u[7], u[4], u[5]};
            ok = rotation_form(ux, pp.rot_min_c, q, &fr, &fi);
            lead_x = ok;
          }
          const double nr = sr * fr - si * fi, ni = sr * fi + si * fr;
          // the stored amplitudes grow by 1 / |scalar| within the sweep: keep the
          // matrix form once the sweep's own scalar would drop below the floor
          if (ok && std::hypot(nr, ni) < pp.scale_floor) ok = false;
          if (ok) {
            rot.push_back(i);
            if (lead_x) xrot.push_back(i);
            qs.insert(qs.end(), q, q + 5);
            sr = nr;
            si = ni;
          } else {
            mat.push_back(i);
          }
        }
        if (!rot.empty()) {
          emit_rotation(rot, qs, xrot);
          sw.scale_re = sr;
          sw.scale_im = si;
        }
        if (!mat.empty()) emit_matrix(mat);
        run.clear();
        run_ops.clear();
      };
      for (int32_t li : stage_list[s].second) {
        const PGate& pg = gates[list[li]];
        if (folded[li]) {
          // compose the register map of the permutation onto the exit permutation
          const int ta = reg_of_pos[pos_of[pg.q0]];
          int cb = -1, sb = -1;
          if (pg.kind == PK_SWAP) sb = reg_of_pos[pos_of[pg.q1]];
          else if (pg.cmask) cb = reg_of_pos[pos_of[__builtin_ctzll(pg.cmask)]];
          for (int j = 0; j < (1 << NR); ++j) {
            int x = st.perm[j];
            if (pg.kind == PK_SWAP) {
              const int ba = (x >> ta) & 1, bb = (x >> sb) & 1;
              if (ba != bb) x ^= (1 << ta) | (1 << sb);
            } else if (cb < 0 || ((x >> cb) & 1)) {
              x ^= 1 << ta;
            }
            st.perm[j] = (int8_t)x;
          }
          folded_bits |= 1u << ta;
          if (cb >= 0) folded_bits |= 1u << cb;
          if (sb >= 0) folded_bits |= 1u << sb;
          folded_ops.push_back(pg.op_index);
          continue;
        }
        if (pg.kind == PK_DENSE1 && pg.cmask == 0) {
          const int bit = reg_of_pos[pos_of[pg.q0]];
          for (const auto& r : run)
            if (r.first == bit) {
              flush_run();
              break;
            }
          run.emplace_back(bit, pg.m);
          run_ops.push_back(pg.op_index);
          continue;
        }
        flush_run();
        SwGate sg;
        std::memset(&sg, 0, sizeof sg);
        for (uint64_t m = pg.cmask; m; m &= m - 1) {
          const int c = __builtin_ctzll(m);
          if (pos_of[c] >= 0) sg.lmask |= 1u << pos_of[c];
          else sg.gmask |= 1ULL << phys_of[c];
        }
        auto ref = [&](int q) { return pos_of[q] >= 0 ? pos_of[q] : -phys_of[q] - 1; };
        sg.moff = (int32_t)plan.pool.size();
        switch (pg.kind) {
          case PK_DENSE1:
            sg.kind = SK_G1;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            plan.pool.insert(plan.pool.end(), pg.m, pg.m + 8);
            break;
          case PK_DENSE2:
            sg.kind = SK_G2;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            sg.b = reg_of_pos[pos_of[pg.q1]];
            plan.pool.insert(plan.pool.end(), pg.m, pg.m + 32);
            break;
          case PK_X: {
            sg.kind = SK_X;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            // a control that is a register bit turns the gate into a register permutation
            for (uint64_t m = pg.cmask; m; m &= m - 1) {
              const int c = __builtin_ctzll(m);
              if (pos_of[c] >= 0 && reg_of_pos[pos_of[c]] >= 0) {
                // the remaining tile controls must lie outside the registers
                const uint32_t rest = sg.lmask & ~(1u << pos_of[c]);
                if (rest & R) break;
                sg.kind = SK_CX;
                sg.b = reg_of_pos[pos_of[c]];
                sg.lmask = rest;
                break;
              }
            }
            break;
          }
          case PK_SWAP:
            sg.kind = SK_SWAP;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            sg.b = reg_of_pos[pos_of[pg.q1]];
            break;
          case PK_PAULI:
            sg.kind = SK_PAULI;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            sg.b = pg.q1;  // slot
            break;
          case PK_TMAT:
            sg.kind = SK_TMAT;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            sg.b = pg.q1;  // Kraus point
            break;
          case PK_PROBE:
            sg.kind = SK_PROBE;
            sg.a = reg_of_pos[pos_of[pg.q0]];
            sg.b = (int32_t)pg.op_index;  // gradient slot
            break;
          case PK_DIAG1:
            sg.kind = SK_D1;
            sg.a = ref(pg.q0);
            if (pg.cmask == 0 && sg.a >= 0 && reg_of_pos[sg.a] >= 0) {
              sg.kind = SK_D1R;
              sg.a = reg_of_pos[sg.a];
              const double n0 = pg.m[0] * pg.m[0] + pg.m[1] * pg.m[1];
              if (pp.phase_free && n0 > 0.0) {
                // diag(d0, d1) = d0 diag(1, d1 / d0); the phase-free plan keeps the second
                sg.kind = SK_D1H;
                const double dr = (pg.m[2] * pg.m[0] + pg.m[3] * pg.m[1]) / n0;
                const double di = (pg.m[3] * pg.m[0] - pg.m[2] * pg.m[1]) / n0;
                // |d0| = 1 for the unitaries of a gradient plan; anything else keeps d0
                if (std::fabs(n0 - 1.0) <= 1e-13) {
                  plan.pool.push_back(dr);
                  plan.pool.push_back(di);
                  break;
                }
                sg.kind = SK_D1R;
              }
            }
            plan.pool.insert(plan.pool.end(), pg.m, pg.m + 4);
            break;
          case PK_DIAG2: {
            sg.a = ref(pg.q0);
            sg.b = ref(pg.q1);
            if (is_parity_diag(pg)) {
              sg.kind = SK_DP;
              if (sg.a >= 0 && sg.b >= 0 && reg_of_pos[sg.a] >= 0 && reg_of_pos[sg.b] >= 0) {
                sg.kind = SK_DPR;
                sg.a = reg_of_pos[sg.a];
                sg.b = reg_of_pos[sg.b];
              }
              plan.pool.insert(plan.pool.end(), pg.m, pg.m + 4);
            } else {
              sg.kind = SK_D2;
              plan.pool.insert(plan.pool.end(), pg.m, pg.m + 8);
            }
            break;
          }
        }
        if (sg.kind == SK_X && sg.lmask == 0) sg.kind = SK_X0;
        if (sg.kind == SK_CX && sg.lmask == 0) sg.kind = SK_CX0;
        sg.code = sg.kind == SK_PROBE ? (SK_PROBE << 4) | (sg.a << 2) | (pg.q1 & 3)
                                      : sw_code(sg.kind, sg.a, sg.b);
        plan.gates.push_back(sg);
        plan.gate_ops.push_back(pg.op_index);
      }
      flush_run();
      if (pp.peephole)
        optimize_stage(plan, st.g0, st, reg_of_pos, folded_bits, is_last, &sw.scale_re,
                       &sw.scale_im);
      merge_register_diagonals(plan, st.g0, NR, (size_t)sw.pool0 + (size_t)pp.max_pool);
      plan.gate_ops.insert(plan.gate_ops.end(), folded_ops.begin(), folded_ops.end());
      st.g1 = (int32_t)plan.gates.size();
      StageEntry en;
      en.g_start = st.g0;
      if (pp.entry_fold) fold_stage_entry(plan, st, &en);
      plan.stages.push_back(st);
      plan.entry.push_back(en);
    }
    sw.s1 = (int32_t)plan.stages.size();
    sw.pool1 = (int32_t)plan.pool.size();
    plan.sweeps.push_back(sw);
    // the layout after this sweep
    for (int p = 0; p < T; ++p) {
      const int q = log_at[p];
      phys_of[q] = sw.outp[p];
      log_of[sw.outp[p]] = q;
    }

    for (int32_t g : list) idx_in_sweep[g] = -1;
    ++sweep_id;
    while (first < G && when[first] >= 0) ++first;
  }
  plan.restore = restore_identity(phys_of, n);

  // A scalar commutes with every gate, so the sweeps' rotation-form scalars need not
  // be applied where they arise: carry their product on and apply it at the store of
  // the last sweep, or earlier once its magnitude drops below the floor.
  double cr = 1.0, ci = 0.0;
  for (size_t k = 0; k < plan.sweeps.size(); ++k) {
    SwSweep& sw = plan.sweeps[k];
    const double nr = cr * sw.scale_re - ci * sw.scale_im;
    const double ni = cr * sw.scale_im + ci * sw.scale_re;
    cr = nr;
    ci = ni;
    if (k + 1 == plan.sweeps.size() || std::hypot(cr, ci) < pp.scale_floor) {
      sw.scale_re = cr;
      sw.scale_im = ci;
      cr = 1.0;
      ci = 0.0;
    } else {
      sw.scale_re = 1.0;
      sw.scale_im = 0.0;
    }
  }
  return plan;
}

}  // namespace sc
