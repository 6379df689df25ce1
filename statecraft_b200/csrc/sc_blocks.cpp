// Dense-block cutting (host): runs of gates on at most 5 qubits composed into one
// unitary for the FP64 tensor-core kernel (k_block.cu).
//
// The gate stream is walked in order.  A block collects consecutive gates while the
// union of the qubits they touch stays within 5; the gate that does not fit closes
// it.  A closed block is kept when it touches at least 3 qubits (the smallest tile
// of the tensor-core kernel is 8 x 8) and its gates' summed cost (gate_cost: FP
// multiply-adds per amplitude on the sweep path) reaches the threshold; otherwise its
// gates return to the sweep-planned stream.  The block's unitary is the product of
// its gates in the 2^k-dimensional space of its qubits (local bit b <-> the b-th
// qubit in ascending order), built column by column: each gate acts on every column
// of the running product, U <- G U.
#include <algorithm>
#include <complex>
#include <cstring>

#include "sc_internal.h"

namespace sc {

namespace {

using cd = std::complex<double>;

bool blockable(const PGate& g) {
  switch (g.kind) {
    case PK_DENSE1: case PK_DENSE2: case PK_X: case PK_SWAP: case PK_DIAG1: case PK_DIAG2:
      return true;
    default:
      return false;
  }
}

// applies g to a vector over the block's local basis (dim = 2^k)
void apply_local(const PGate& g, const int* local_of, int dim, cd* v) {
  auto bit = [&](int q) { return 1 << local_of[q]; };
  int cm = 0;
  for (uint64_t m = g.cmask; m; m &= m - 1) cm |= bit(__builtin_ctzll(m));
  auto c = [&](int k) { return cd(g.m[2 * k], g.m[2 * k + 1]); };
  switch (g.kind) {
    case PK_DENSE1: {
      const int t = bit(g.q0);
      for (int i = 0; i < dim; ++i) {
        if ((i & t) || (i & cm) != cm) continue;
        const cd a0 = v[i], a1 = v[i | t];
        v[i] = c(0) * a0 + c(1) * a1;
        v[i | t] = c(2) * a0 + c(3) * a1;
      }
      break;
    }
    case PK_DENSE2: {  // local index 2 * bit(first) + bit(second)
      const int f = bit(g.q0), s = bit(g.q1);
      for (int i = 0; i < dim; ++i) {
        if (i & (f | s)) continue;
        const int idx[4] = {i, i | s, i | f, i | f | s};
        cd a[4], o[4];
        for (int r = 0; r < 4; ++r) a[r] = v[idx[r]];
        for (int r = 0; r < 4; ++r) {
          o[r] = 0.0;
          for (int q = 0; q < 4; ++q) o[r] += c(4 * r + q) * a[q];
        }
        for (int r = 0; r < 4; ++r) v[idx[r]] = o[r];
      }
      break;
    }
    case PK_X: {
      const int t = bit(g.q0);
      for (int i = 0; i < dim; ++i)
        if (!(i & t) && (i & cm) == cm) std::swap(v[i], v[i | t]);
      break;
    }
    case PK_SWAP: {
      const int a = bit(g.q0), b = bit(g.q1);
      for (int i = 0; i < dim; ++i)
        if ((i & a) && !(i & b)) std::swap(v[i], v[(i & ~a) | b]);
      break;
    }
    case PK_DIAG1: {
      const int t = bit(g.q0);
      for (int i = 0; i < dim; ++i)
        if ((i & cm) == cm) v[i] *= (i & t) ? c(1) : c(0);
      break;
    }
    case PK_DIAG2: {
      const int f = bit(g.q0), s = bit(g.q1);
      for (int i = 0; i < dim; ++i) v[i] *= c(2 * ((i & f) ? 1 : 0) + ((i & s) ? 1 : 0));
      break;
    }
    default: break;
  }
}

DenseBlock compose(const std::vector<PGate>& gs, uint64_t qmask) {
  DenseBlock b;
  std::memset(&b.args, 0, sizeof b.args);
  b.n_gates = (int32_t)gs.size();
  int local_of[64];
  for (int q = 0; q < 64; ++q) local_of[q] = -1;
  for (uint64_t m = qmask; m; m &= m - 1) {
    const int q = __builtin_ctzll(m);
    local_of[q] = b.args.k;
    b.args.q[b.args.k++] = q;
  }
  const int dim = 1 << b.args.k;
  std::vector<cd> u((size_t)dim * dim, 0.0);  // column-major while composing
  for (int j = 0; j < dim; ++j) u[(size_t)j * dim + j] = 1.0;
  for (const PGate& g : gs)
    for (int j = 0; j < dim; ++j) apply_local(g, local_of, dim, &u[(size_t)j * dim]);
  b.u.resize(2 * (size_t)dim * dim);
  for (int r = 0; r < dim; ++r)
    for (int j = 0; j < dim; ++j) {
      b.u[2 * ((size_t)r * dim + j)] = u[(size_t)j * dim + r].real();
      b.u[2 * ((size_t)r * dim + j) + 1] = u[(size_t)j * dim + r].imag();
    }
  return b;
}

}  // namespace

std::vector<GateRun> cut_dense_blocks(const std::vector<PGate>& gates, int n, double min_cost,
                                      std::vector<DenseBlock>* blocks) {
  std::vector<GateRun> out(1);
  std::vector<PGate> cur;
  uint64_t cur_mask = 0;
  double cur_cost = 0.0;
  auto close = [&]() {
    const int k = __builtin_popcountll(cur_mask);
    if (!cur.empty() && k >= 3 && k <= 5 && n >= k + 3 && cur_cost >= min_cost) {
      blocks->push_back(compose(cur, cur_mask));
      out.back().block = (int)blocks->size() - 1;
      out.emplace_back();
    } else {
      out.back().gates.insert(out.back().gates.end(), cur.begin(), cur.end());
    }
    cur.clear();
    cur_mask = 0;
    cur_cost = 0.0;
  };
  for (const PGate& g : gates) {
    if (!blockable(g)) {
      close();
      out.back().gates.push_back(g);
      continue;
    }
    const uint64_t t = touch_mask(g);
    if (__builtin_popcountll(cur_mask | t) > 5) close();
    if (__builtin_popcountll(t) > 5) {  // e.g. a gate with many controls
      out.back().gates.push_back(g);
      continue;
    }
    cur.push_back(g);
    cur_mask |= t;
    cur_cost += gate_cost(g);
  }
  close();
  if (out.back().gates.empty() && out.back().block < 0) out.pop_back();
  return out;
}

}  // namespace sc
