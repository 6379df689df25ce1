// Fused tile-sweep kernel: one HBM read + one HBM write of every amplitude
// applies every gate the planner packed into the sweep.
//
// Tile: the 2^T amplitudes whose indices differ only in the tile qubits (the L
// lowest qubits, contiguous in memory, plus h high qubits), i.e. 2^h contiguous
// segments of 2^L amplitudes.  A persistent CTA walks tiles with two shared-memory
// tile buffers: while it computes tile i in one buffer, TMA bulk copies
// (cp.async.bulk, one per segment, completing on an mbarrier) stream tile i+1 into
// the other, and the results of tile i drain to HBM as bulk stores.
//
// Per tile the sweep's stages run in registers: in stage s each thread holds 2^NR
// amplitudes that differ in the stage's register positions R[0..NR-1] and applies
// the stage's gates there; the next stage re-distributes the tile through the
// buffer with an XOR swizzle.  The first stage reads and the last stage writes the
// buffer in the linear (TMA) layout; with R on high positions the lanes of a warp
// walk the low positions, so those accesses are conflict-free too.
//
// The whole sweep plan (stages, register tables, gates, matrices) is a
// __grid_constant__ kernel parameter: every thread reads the same record at the
// same time, which the constant cache serves as a broadcast.
//
// Every mbarrier wait is bounded (about a second of clock cycles); on timeout the
// CTA records an error in `err`, waits (bounded) for the copies it issued and
// returns, and the host reports SC_ETIMEOUT.
#include <cuda.h>

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <type_traits>

#include "sc_device.cuh"
#include "sc_internal.h"
#include "sc_sweep.h"

namespace sc {

namespace {

// Tile offsets of a stage's registers: register j sits at local index l0 | off[j],
// off[j] the OR of rb[k] (1 << register position k) over the set bits k of j.
// Kept as NR words, not 2^NR, so the record loop carries fewer registers.
template <int NR>
struct RegOff {
  uint32_t rb[NR];
  __device__ __forceinline__ uint32_t operator[](int j) const {
    uint32_t o = 0;
#pragma unroll
    for (int k = 0; k < NR; ++k)
      if (j & (1 << k)) o |= rb[k];
    return o;
  }
};

// Exit-slot flips of a stage's slot folds: register j leaves through its slot XOR
// x0 XOR (xc[k] for each set bit k of j); the flips are linear in j.
template <int NR>
struct SlotFlips {
  uint32_t x0, xc[NR];
  __device__ __forceinline__ uint32_t operator[](int j) const {
    uint32_t f = x0;
#pragma unroll
    for (int k = 0; k < NR; ++k)
      if (j & (1 << k)) f ^= xc[k];
    return f;
  }
};

// Slot of tile index i in the shared-memory layout a stage reads (its exchange's
// swizzle; the fixed default unless rows[0] bit 15 is set).  Uniform per stage.
template <typename R>
__device__ __forceinline__ uint32_t stage_swz(uint32_t i, const SwStageTab& t) {
  constexpr int K = Amp<R>::kSwizzleShift;
  if (!(t.rows[0] & 0x8000u)) return swz<R>(i);
  uint32_t lo = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) lo |= (__popc(i & (uint32_t)t.rows[k]) & 1u) << k;
  return i ^ lo;
}

template <typename R, int NR, int A_>
__device__ __forceinline__ void g1(typename Amp<R>::type (&v)[1 << NR], const R* m,
                                   uint32_t l0, const RegOff<NR>& off, uint32_t lmask) {
  const R m00r = m[0], m00i = m[1], m01r = m[2], m01i = m[3];
  const R m10r = m[4], m10i = m[5], m11r = m[6], m11i = m[7];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & (1 << A_)) continue;
    const int j1 = j | (1 << A_);
    if (lmask && (((l0 | off[j]) & lmask) != lmask)) continue;
    const auto a0 = v[j], a1 = v[j1];
    // every use of a0 comes before any use of a1 and the last use of a1 completes
    // each output, so the outputs can take the inputs' registers in place
    R o0x = m00r * a0.x, o0y = m00r * a0.y, o1x = m10r * a0.x, o1y = m10r * a0.y;
    o0x = fma(-m00i, a0.y, o0x);
    o0y = fma(m00i, a0.x, o0y);
    o1x = fma(-m10i, a0.y, o1x);
    o1y = fma(m10i, a0.x, o1y);
    o0x = fma(m01r, a1.x, o0x);
    o0y = fma(m01r, a1.y, o0y);
    o1x = fma(m11r, a1.x, o1x);
    o1y = fma(m11r, a1.y, o1y);
    o0x = fma(-m01i, a1.y, o0x);
    o0y = fma(m01i, a1.x, o0y);
    o1x = fma(-m11i, a1.y, o1x);
    o1y = fma(m11i, a1.x, o1y);
    v[j] = make_amp<R>(o0x, o0y);
    v[j1] = make_amp<R>(o1x, o1y);
  }
}

// parity diagonal on register bits A_, B_: factor d[bit A_ ^ bit B_], fixed per register
template <typename R, int NR, int A_, int B_>
__device__ __forceinline__ void dpr(typename Amp<R>::type (&v)[1 << NR], const R* m) {
  const R d0r = m[0], d0i = m[1], d1r = m[2], d1i = m[3];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const int par = ((j >> A_) ^ (j >> B_)) & 1;
    v[j] = par ? cmul(d1r, d1i, v[j]) : cmul(d0r, d0i, v[j]);
  }
}

// 4x4 on register bits (A_ = first, B_ = second); local basis 2*bit(first)+bit(second)
template <typename R, int NR, int A_, int B_>
__device__ __forceinline__ void g2(typename Amp<R>::type (&v)[1 << NR], const R* m) {
  using A = typename Amp<R>::type;
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & ((1 << A_) | (1 << B_))) continue;
    const int idx[4] = {j, j | (1 << B_), j | (1 << A_), j | (1 << A_) | (1 << B_)};
    A a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = v[idx[k]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      A o;
      o.x = 0;
      o.y = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const R mr = m[2 * (4 * r + c)], mi = m[2 * (4 * r + c) + 1];
        o.x += mr * a[c].x - mi * a[c].y;
        o.y += mr * a[c].y + mi * a[c].x;
      }
      v[idx[r]] = o;
    }
  }
}

// Diagonals whose bits may lie outside the registers: a tile position (ref >= 0,
// read from the thread's tile index) or a global qubit (ref < 0, fixed per tile).
// diag1: diag(d0, d1) on one bit with tile-position controls lmask.
template <typename R, int NR>
__device__ __forceinline__ void diag1_any(typename Amp<R>::type (&v)[1 << NR], const R* m, int a,
                                          uint32_t l0, const RegOff<NR>& off,
                                          uint32_t lmask, uint32_t base) {
  const uint32_t gb = a < 0 ? ((base >> (-a - 1)) & 1u) : 0u;
  const int sh = a < 0 ? 0 : a;
  const uint32_t lm = a < 0 ? 0u : 1u;
  const R d0r = m[0], d0i = m[1], d1r_ = m[2], d1i_ = m[3];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const uint32_t li = l0 | off[j];
    if ((li & lmask) != lmask) continue;
    const uint32_t bit = ((li >> sh) & lm) | gb;
    v[j] = cmul(bit ? d1r_ : d0r, bit ? d1i_ : d0i, v[j]);
  }
}

// parity diagonal: factor d[bit(a) ^ bit(b)]
template <typename R, int NR>
__device__ __forceinline__ void diagp_any(typename Amp<R>::type (&v)[1 << NR], const R* m, int a,
                                          int bq, uint32_t l0, const RegOff<NR>& off,
                                          uint32_t base) {
  const uint32_t gpar = (a < 0 ? ((base >> (-a - 1)) & 1u) : 0u) ^
                        (bq < 0 ? ((base >> (-bq - 1)) & 1u) : 0u);
  const uint32_t pm = (a < 0 ? 0u : (1u << a)) | (bq < 0 ? 0u : (1u << bq));
  const R d0r = m[0], d0i = m[1], d1r_ = m[2], d1i_ = m[3];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const uint32_t bit = (__popc((l0 | off[j]) & pm) & 1u) ^ gpar;
    v[j] = cmul(bit ? d1r_ : d0r, bit ? d1i_ : d0i, v[j]);
  }
}

// general two-bit diagonal, factor d[2 bit(a) + bit(b)]
template <typename R, int NR>
__device__ __forceinline__ void diag2_any(typename Amp<R>::type (&v)[1 << NR], const R* m, int a,
                                          int bq, uint32_t l0, const RegOff<NR>& off,
                                          uint32_t base) {
  const uint32_t ga = a < 0 ? ((base >> (-a - 1)) & 1u) : 0u;
  const uint32_t gbb = bq < 0 ? ((base >> (-bq - 1)) & 1u) : 0u;
  const int sa = a < 0 ? 0 : a, sb = bq < 0 ? 0 : bq;
  const uint32_t ma = a < 0 ? 0u : 1u, mb = bq < 0 ? 0u : 1u;
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const uint32_t li = l0 | off[j];
    const uint32_t k = ((((li >> sa) & ma) | ga) << 1) | (((li >> sb) & mb) | gbb);
    v[j] = cmul(m[2 * k], m[2 * k + 1], v[j]);
  }
}

// X on register bit A_ applied to the stage's exit slots: the amplitude in register
// j leaves through the slot of register j ^ (1 << A_), whose swizzled offset differs
// by m = xoff[A_], the slot offset of that bit (the offsets are linear in j); m = 0 where the gate's
// controls outside the registers are not all set
template <int NR, int A_>
__device__ __forceinline__ void xfold(SlotFlips<NR>& fl, uint32_t m) {
  fl.x0 ^= m;
}

// the same for X on register bit T_ controlled by register bit C_
template <int NR, int T_, int C_>
__device__ __forceinline__ void cxfold(SlotFlips<NR>& fl, uint32_t m) {
  fl.xc[C_] ^= m;
}

// uncontrolled diag(d0, d1) on register bit A_: the factor of each register is fixed
template <typename R, int NR, int A_>
__device__ __forceinline__ void d1r(typename Amp<R>::type (&v)[1 << NR], const R* m) {
  const R d0r = m[0], d0i = m[1], d1r_ = m[2], d1i_ = m[3];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j)
    v[j] = ((j >> A_) & 1) ? cmul(d1r_, d1i_, v[j]) : cmul(d0r, d0i, v[j]);
}

// Rotation form of commuting 2x2 gates on the register bits of mask M: each gate is
// diag(1, e^{i phi}) [[1, -t], [t, 1]] diag(1, e^{i lam}) (its scalar is applied by
// the sweep), and since the gates act on distinct bits their input and output
// phases combine into one diagonal each.  Pool: t per bit (ascending), t / (1 + t^2)
// per bit, then the input-phase table lam[s] (which also carries the real factors
// 1 + t^2 of the bits in s) and the output-phase table phi[s], complex, for
// s = 1 .. 2^K - 1 (s = the bits of j in M, compacted; s = 0 is the phase 1).
// A 4-bit record costs 15 + 15 complex multiplies and 4 x 8 rotations (248 FP64
// operations for 16 amplitudes, all in place) where four single-bit gates cost 384.
template <int M>
__host__ __device__ constexpr int compact_bits(int j) {
  int s = 0, k = 0;
  for (int b = 0; b < 4; ++b)
    if ((M >> b) & 1) s |= ((j >> b) & 1) << k++;
  return s;
}

// [[1, -t], [t, 1]] on register bit A_ as two shears, the amplitude on the 1 side
// arriving scaled by 1 + t^2 (the record's input table): a0 -= tp a1, a1 += t a0 with
// tp = t / (1 + t^2).  Each update overwrites the value it reads last, so the pair
// stays in its registers (no temporaries to move back at the record's end).
template <typename R, int NR, int A_>
__device__ __forceinline__ void rot(typename Amp<R>::type (&v)[1 << NR], const R t, const R tp) {
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & (1 << A_)) continue;
    const int j1 = j | (1 << A_);
    v[j].x = fma(-tp, v[j1].x, v[j].x);
    v[j].y = fma(-tp, v[j1].y, v[j].y);
    v[j1].x = fma(t, v[j].x, v[j1].x);
    v[j1].y = fma(t, v[j].y, v[j1].y);
  }
}

template <typename R, int NR, int M>
__device__ __forceinline__ void phase_table(typename Amp<R>::type (&v)[1 << NR], const R* tab) {
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const int s = compact_bits<M>(j);
    if (s != 0) v[j] = cmul(tab[2 * (s - 1)], tab[2 * (s - 1) + 1], v[j]);
  }
}

template <typename R, int NR, int M>
__device__ __forceinline__ void g1allq(typename Amp<R>::type (&v)[1 << NR], const R* q) {
  constexpr int K = ((M >> 0) & 1) + ((M >> 1) & 1) + ((M >> 2) & 1) + ((M >> 3) & 1);
  const R* lam = q + 2 * K;
  const R* phi = lam + 2 * ((1 << K) - 1);
  phase_table<R, NR, M>(v, lam);
  const R* tq = q;
  if constexpr ((M & 1) != 0) { rot<R, NR, 0>(v, tq[0], tq[K]); ++tq; }
  if constexpr (NR > 1 && (M & 2) != 0) { rot<R, NR, 1>(v, tq[0], tq[K]); ++tq; }
  if constexpr (NR > 2 && (M & 4) != 0) { rot<R, NR, 2>(v, tq[0], tq[K]); ++tq; }
  if constexpr (NR > 3 && (M & 8) != 0) rot<R, NR, 3>(v, tq[0], tq[K]);
  phase_table<R, NR, M>(v, phi);
}

// uncontrolled 2x2 gates on the register bits of mask M (ascending; matrices
// consecutive in the pool)
template <typename R, int NR, int M>
__device__ __forceinline__ void g1all(typename Amp<R>::type (&v)[1 << NR], const R* m,
                                      uint32_t l0, const RegOff<NR>& off) {
  const R* mm = m;
  if constexpr ((M & 1) != 0) {
    g1<R, NR, 0>(v, mm, l0, off, 0u);
    mm += 8;
  }
  if constexpr (NR > 1 && (M & 2) != 0) {
    g1<R, NR, 1>(v, mm, l0, off, 0u);
    mm += 8;
  }
  if constexpr (NR > 2 && (M & 4) != 0) {
    g1<R, NR, 2>(v, mm, l0, off, 0u);
    mm += 8;
  }
  if constexpr (NR > 3 && (M & 8) != 0) g1<R, NR, 3>(v, mm, l0, off, 0u);
}

// real rotations on the register bits of mask M as lifting shears (pool: p, s per
// bit, ascending): a0 += p a1, a1 += s a0, a0 += p a1, every update in place
template <typename R, int NR, int M>
__device__ __forceinline__ void rotl(typename Amp<R>::type (&v)[1 << NR], const R* q) {
#pragma unroll
  for (int b = 0, k = 0; b < NR; ++b) {
    if (!((M >> b) & 1)) continue;
    const R pp = q[2 * k], ss = q[2 * k + 1];
    ++k;
#pragma unroll
    for (int j = 0; j < (1 << NR); ++j) {
      if (j & (1 << b)) continue;
      const int j1 = j | (1 << b);
      v[j].x = fma(pp, v[j1].x, v[j].x);
      v[j].y = fma(pp, v[j1].y, v[j].y);
      v[j1].x = fma(ss, v[j].x, v[j1].x);
      v[j1].y = fma(ss, v[j].y, v[j1].y);
      v[j].x = fma(pp, v[j1].x, v[j].x);
      v[j].y = fma(pp, v[j1].y, v[j].y);
    }
  }
}

// diag(1, d) on register bit A_: only the registers with the bit set change
template <typename R, int NR, int A_>
__device__ __forceinline__ void d1h(typename Amp<R>::type (&v)[1 << NR], const R* m) {
  const R dr = m[0], di = m[1];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j)
    if ((j >> A_) & 1) v[j] = cmul(dr, di, v[j]);
}

// diagonal over the register bits as a table: register j times entry j
template <typename R, int NR>
__device__ __forceinline__ void dtab(typename Amp<R>::type (&v)[1 << NR], const R* m) {
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) v[j] = cmul(m[2 * j], m[2 * j + 1], v[j]);
}

// A register permutation applied through the thread's own shared-memory slots:
// register j goes out to the slot it was read from in this stage (rbase ^ rd[j])
// and comes back from the slot of its source register, rbase ^ src_rd(j) (the rd
// entry of the source; conditions select between entries, so every constant load
// has an index common to the warp).  The slots belong to this thread alone from the
// stage's read to the next exchange, so no barrier is needed.  Done in registers, a
// permutation chosen at run time makes the record's code move the amplitude
// registers back into place where the record loop joins.
template <typename A, int NV, typename F>
__device__ __forceinline__ void smem_permute(A (&v)[NV], A* cur, uint32_t rbase,
                                             const SwStageTab& tab, F&& src_rd) {
#pragma unroll
  for (int j = 0; j < NV; ++j) cur[rbase ^ tab.rd[j]] = v[j];
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = cur[rbase ^ (uint32_t)src_rd(j)];
}

// Pauli chosen per trajectory on register bit A_ (1 = X, 2 = Y, 3 = Z; the identity
// never reaches here).  Z negates in place; X and Y move the pair through the
// thread's own slots (smem_permute), Y taking the components crosswise on the way
// back: new0 = -i a1 = (a1.y, -a1.x), new1 = i a0 = (-a0.y, a0.x).
template <typename R, int NR, int A_>
__device__ __forceinline__ void pauli_slots(typename Amp<R>::type (&v)[1 << NR], uint32_t code,
                                            typename Amp<R>::type* cur, uint32_t rbase,
                                            const SwStageTab& tab) {
  if (code == 3u) {
#pragma unroll
    for (int j = 0; j < (1 << NR); ++j)
      if ((j >> A_) & 1) v[j] = make_amp<R>(-v[j].x, -v[j].y);
    return;
  }
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) cur[rbase ^ tab.rd[j]] = v[j];
  const uint32_t c = code == 2u ? 1u : 0u;  // Y: components crosswise
  const R sg = code == 2u ? (R)-1 : (R)1;
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const R* sp = reinterpret_cast<const R*>(cur + (rbase ^ tab.rd[j ^ (1 << A_)]));
    const R c0 = sp[c], c1 = sp[c ^ 1u];
    if ((j >> A_) & 1) {
      v[j].x = sg * c0;
      v[j].y = c1;
    } else {
      v[j].x = c0;
      v[j].y = sg * c1;
    }
  }
}

// Pauli slot conjugated through folded register permutations: i^p X^u Z^w over the
// register bits, f = (u, w, p) of the trajectory's choice.  Register j takes
// i^p (-1)^{|w & (j ^ u)|} times register j ^ u, through the thread's own slots (the
// i^p taken as a component swap and signs on the way back).
template <typename R, int NR>
__device__ __forceinline__ void pauli_frame_slots(typename Amp<R>::type (&v)[1 << NR], const R* f,
                                                  typename Amp<R>::type* cur, uint32_t rbase,
                                                  const SwStageTab& tab) {
  const uint32_t u = (uint32_t)f[0], w = (uint32_t)f[1], ph = (uint32_t)f[2] & 3u;
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) cur[rbase ^ tab.rd[j]] = v[j];
  const uint32_t c = ph & 1u;  // odd powers of i swap the components
  const R sx = (ph == 1u || ph == 2u) ? (R)-1 : (R)1;
  const R sy = (ph >= 2u) ? (R)-1 : (R)1;
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const uint32_t src = ((uint32_t)j ^ u) & ((1u << NR) - 1u);
    const R* sp = reinterpret_cast<const R*>(cur + (rbase ^ tab.rd[src]));
    const R sw = (__popc(w & src) & 1) ? (R)-1 : (R)1;
    v[j].x = (sx * sw) * sp[c];
    v[j].y = (sy * sw) * sp[c ^ 1u];
  }
}

// switch cases for the dispatch code (sw_code): one jump per gate into code that
// is specialised on its register bits
#define SC_CASE_1(K, A, F) \
  case ((K) << 4) | ((A) << 2):  \
    if constexpr ((A) < NR) {    \
      F(A);                      \
    }                            \
    break;
#define SC_CASES_1(K, F) SC_CASE_1(K, 0, F) SC_CASE_1(K, 1, F) SC_CASE_1(K, 2, F) SC_CASE_1(K, 3, F)
#define SC_CASE_2(K, A, B, F)              \
  case ((K) << 4) | ((A) << 2) | (B):      \
    if constexpr ((A) < NR && (B) < NR) {  \
      F(A, B);                             \
    }                                      \
    break;
#define SC_CASES_2(K, F)                                                                  \
  SC_CASE_2(K, 0, 1, F) SC_CASE_2(K, 0, 2, F) SC_CASE_2(K, 0, 3, F) SC_CASE_2(K, 1, 0, F) \
  SC_CASE_2(K, 1, 2, F) SC_CASE_2(K, 1, 3, F) SC_CASE_2(K, 2, 0, F) SC_CASE_2(K, 2, 1, F) \
  SC_CASE_2(K, 2, 3, F) SC_CASE_2(K, 3, 0, F) SC_CASE_2(K, 3, 1, F) SC_CASE_2(K, 3, 2, F)

// tile position bits -> physical offset in the input layout (host, sweep parameters)
template <typename P>
uint64_t host_spread_t(uint64_t x, const P& p) {
  uint64_t g = x & ((1ULL << p.L) - 1ULL);
  uint64_t hi = x >> p.L;
  for (int k = 0; hi; ++k, hi >>= 1)
    if (hi & 1ULL) g |= 1ULL << p.hq[k];
  return g;
}

// local tile index -> global offset (n <= 32: 32-bit)
template <typename P>
__device__ __forceinline__ uint32_t spread32(uint32_t x, const P& p) {
  uint32_t g = x & ((1u << p.L) - 1u);
  uint32_t hi = x >> p.L;
#pragma unroll 1
  for (int k = 0; hi; ++k, hi >>= 1)
    if (hi & 1u) g |= 1u << p.hq[k];
  return g;
}

// the thread's index bits placed around the stage's register positions
template <int NR>
__device__ __forceinline__ uint32_t stage_l0(uint32_t tid, const SwStage& s) {
  uint32_t x = tid;
#pragma unroll
  for (int k = 0; k < NR; ++k) x = insert_zero32(x, s.R[k]);
  return x;
}

// tile position bits -> physical offset in the output layout
template <typename P>
__device__ __forceinline__ uint32_t spread_out32(uint32_t x, const P& p) {
  uint32_t g = 0;
#pragma unroll 1
  for (int k = 0; x; ++k, x >>= 1)
    if (x & 1u) g |= 1u << p.outp[k];
  return g;
}

// physical offset of tile t: its index bits spread over the non-tile bits
template <typename P>
__host__ __device__ __forceinline__ uint32_t tile_base(uint32_t t, const P& p) {
  uint32_t base = t << p.L;
#pragma unroll 1
  for (int k = 0; k < p.h; ++k) base = insert_zero32(base, p.hs[k]);
  return base;
}

// Register caps.  complex128 NR = 3: 96 registers let five 128-thread CTAs share an
// SM (measured a few percent faster than the uncapped 128).  complex128 NR = 4: 168
// (three CTAs per SM, the limit the two 32 KB tile buffers set anyway).
#ifndef SC_SWEEP_C128_NR3_REGS
#define SC_SWEEP_C128_NR3_REGS 96
#endif
#ifndef SC_SWEEP_C128_NR4_REGS
#define SC_SWEEP_C128_NR4_REGS 168
#endif

template <typename R, int NR>
constexpr int sweep_max_threads() {
  return NR >= 4 ? (sizeof(R) == 8 ? 256 : 512) : (NR == 3 ? 512 : 1024);
}

template <typename R, int NR>
constexpr int sweep_max_regs() {
  return NR == 3 && sizeof(R) == 8   ? SC_SWEEP_C128_NR3_REGS
         : NR == 4 && sizeof(R) == 8 ? SC_SWEEP_C128_NR4_REGS
                                     : std::min(255, 65536 / sweep_max_threads<R, NR>());
}

constexpr long long kWaitLimitCycles = 2000000000LL;  // ~1 s at 2 GHz

// two tile buffers, the two mbarriers of the tile copies (64 bytes), and the Pauli
// choices of a batched sweep's slots (128 bytes)
template <typename R>
__host__ __device__ constexpr size_t sweep_smem_bytes(int T) {
  return 2 * (sizeof(typename Amp<R>::type) << T) + 64 + 128;
}

// One fused sweep.  Persistent CTAs walk the work items (tiles; (state, tile) pairs
// of a batch), double-buffering them in shared memory: while tile i is computed in
// one buffer, tile i + grid arrives in the other -- as one bulk tensor copy (TMA)
// issued by thread 0 and completing on that buffer's mbarrier when kTma (the tile is
// a box of the state tensor), else as per-thread cp.async copies of each thread's
// first-stage registers.  The registers stay live from stage to stage (each stage
// boundary: the previous stage's registers go to their slots in this stage's
// layout, then this stage's registers are read), and results leave from the last
// stage as direct 128-/64-bit stores.  kBatch: the sweep runs over p.batch states
// back to back and Pauli slots read the trajectory's choices, staged in shared
// memory.
template <typename R, int NR, bool kTma, bool kBatch>
__global__ void __launch_bounds__(sweep_max_threads<R, NR>())
    __maxnreg__((sweep_max_regs<R, NR>()))
    k_sweep(typename Amp<R>::type* __restrict__ st, const __grid_constant__ SweepParams<R> p,
            int* __restrict__ err) {
  using A = typename Amp<R>::type;
  constexpr int NV = 1 << NR;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t tile_amps = 1u << p.T;
  A* const buf0 = reinterpret_cast<A*>(smem_raw);
  A* const buf1 = buf0 + tile_amps;
  uint64_t* const bars = reinterpret_cast<uint64_t*>(buf1 + tile_amps);
  // Pauli choices of the current trajectory for this sweep's slots
  uint8_t* const codes = reinterpret_cast<uint8_t*>(bars + 8);
  const uint32_t tid = threadIdx.x;
  const int ns = p.n_stages;
  const uint32_t tile_bytes = tile_amps * (uint32_t)sizeof(A);
  // work items: (state, tile) pairs, tile-major within a state; one state unless
  // the sweep runs over a batch of trajectories
  const uint32_t tiles = kBatch ? (uint32_t)(p.tiles * p.batch) : (uint32_t)p.tiles;
  const uint32_t tile_mask = kBatch ? (uint32_t)p.tiles - 1u : 0xffffffffu;
  auto item_state = [&](uint32_t it) -> A* {
    if constexpr (kBatch) return st + ((uint64_t)(it >> p.tiles_log2) << p.nq);
    return st;
  };
  uint32_t codes_for = 0xffffffffu;

  if constexpr (kTma) {
    if (tid == 0) {
      mbar_init(&bars[0], 1);
      mbar_init(&bars[1], 1);
      mbar_init(&bars[2], 1);  // arrived on by nobody: the test hook's wait
      mbar_init_fence();
    }
    __syncthreads();
  }
  // thread 0 issues a whole tile as one tensor copy (box coordinates of work item it)
  auto issue_load = [&](uint32_t it, int b) {
    int32_t c[kTileTensorMaxRank];
#pragma unroll
    for (int k = 0; k < kTileTensorMaxRank; ++k)
      c[k] = (int32_t)((it >> p.tm_shift[k]) & p.tm_mask[k]);
    mbar_arrive_expect_tx(&bars[b], tile_bytes);
    tensor_load(b ? buf1 : buf0, p.tmap, c, p.tm_rank, &bars[b]);
  };

  // first (load) and last (store) register layouts are tile-invariant
  const uint32_t l0_first = stage_l0<NR>(tid, p.stages[0]);
  const uint32_t l0_last = stage_l0<NR>(tid, p.stages[ns - 1]);
  const uint32_t gt_first = kTma ? 0u : spread32(l0_first, p);
  const uint32_t gt_last = spread_out32(l0_last, p);

  // direct path: each thread copies the amplitudes of its own first-stage registers
  // of the next tile into the other buffer with cp.async while this tile computes
  auto prefetch_own = [&](uint32_t tt, A* dst) {
    const A* src = item_state(tt) + tile_base(tt & tile_mask, p);
#pragma unroll
    for (int j = 0; j < NV; ++j)
      cp_async<sizeof(A)>(dst + (l0_first | p.off0[j]), src + (gt_first | p.gfirst[j]));
  };

  uint32_t t = blockIdx.x;
  uint32_t i = 0;
  // a tile copy that did not land within the wait limit: the error flag is set and
  // the thread stops waiting (it finishes its tiles on whatever the buffer holds, so
  // every barrier is still reached by the whole CTA)
  bool timed_out = false;
  uint32_t issued = 0;  // thread 0: tile copies issued so far (item i of this CTA is copy i)
  if constexpr (kTma) {
    if (tid == 0 && t < tiles) {
      issue_load(t, 0);
      issued = 1;
    }
  } else {
    if (t < tiles) prefetch_own(t, buf0);
    cp_async_commit();
  }
  for (; t < tiles; t += gridDim.x, ++i) {
    const int b = (int)(i & 1u);
    A* const cur = b ? buf1 : buf0;
    __syncthreads();  // every thread is done with the other buffer (last tile's reads)
    const uint32_t tn = t + gridDim.x;
    if constexpr (kTma) {
      if (tid == 0 && tn < tiles && !timed_out) {
        issue_load(tn, b ^ 1);
        issued = i + 2;
      }
      const bool stall = p.stall_first > 0 && i == 0;
      if (!timed_out && !mbar_wait_bounded(stall ? &bars[2] : &bars[b], stall ? 0u : (i >> 1) & 1u,
                                           stall ? (long long)p.stall_first : kWaitLimitCycles)) {
        timed_out = true;
        atomicExch(err, 1);
      }
    } else {
      if (tn < tiles) prefetch_own(tn, b ? buf0 : buf1);
      cp_async_commit();
      cp_async_wait<1>();  // this thread's copies of the current tile have landed
    }
    const uint32_t base = tile_base(t & tile_mask, p);
    if constexpr (kBatch) {
      const uint32_t traj = t >> p.tiles_log2;
      if (traj != codes_for) {  // uniform: every thread of the CTA works on tile t
        __syncthreads();       // readers of the previous trajectory's choices are done
        for (int k = (int)tid; k < p.n_local_slots; k += (int)blockDim.x)
          codes[k] = p.paulis[(size_t)traj * p.n_slots + p.slot_map[k]];
        __syncthreads();
        codes_for = traj;
      }
    }

    // the read flip of a stage's conditional entry folds, for the thread's stage base
    auto entry_flip = [&](const SwStageTab& tab, uint32_t lbase) -> uint32_t {
      uint32_t f = 0;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (tab.rf_g[k] < 0) continue;
        const SwGate& q = p.gates[tab.rf_g[k]];
        if (((uint64_t)base & q.gmask) == q.gmask && (lbase & q.lmask) == q.lmask) f ^= tab.rf_off[k];
      }
      return f;
    };
    A v[NV];
    // the thread's read base in the current stage: its slots are rbase ^ rd[j]
    uint32_t rbase;
    {
      // both copy paths leave the tile in `cur` in the linear layout
      const SwStageTab& tab = p.tabs[0];
      rbase = l0_first ^ entry_flip(tab, l0_first);
#pragma unroll
      for (int j = 0; j < NV; ++j) v[j] = cur[rbase ^ tab.rd[j]];
    }
    uint32_t l0 = l0_first, psw0 = 0;
    RegOff<NR> off;
    SlotFlips<NR> sidx;
#pragma unroll 1
    for (int s = 0; s < ns; ++s) {
      const SwStage& stg = p.stages[s];
      const SwStageTab& tab = p.tabs[s];
      const uint32_t nl0 = (s == 0) ? l0_first : stage_l0<NR>(tid, stg);
      if (s > 0) {
        __syncthreads();  // readers of the buffer are done
        // the previous stage's exit slots: its folded permutation (wsoff) and
        // slot folds (sidx) applied, in this stage's layout
        const SwStageTab& ptab = p.tabs[s - 1];
#pragma unroll
        for (int j = 0; j < NV; ++j) cur[psw0 ^ ptab.wsoff[j] ^ sidx[j]] = v[j];
        __syncthreads();
        rbase = stage_swz<R>(nl0, tab) ^ entry_flip(tab, nl0);
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = cur[rbase ^ tab.rd[j]];
      }
      // this stage's exit slots are in the next stage's layout
      psw0 = s + 1 < ns ? stage_swz<R>(nl0, p.tabs[s + 1]) : 0u;
      sidx.x0 = 0u;
#pragma unroll
      for (int k = 0; k < NR; ++k) sidx.xc[k] = 0u;
      l0 = nl0;
#pragma unroll
      for (int k = 0; k < NR; ++k) off.rb[k] = 1u << stg.R[k];
      // a leading X of the stage's only rotation record is folded into tab.rd
      const uint32_t folded_x = (uint32_t)tab.xm;

#pragma unroll 1
      for (int gi = stg.g0;; ++gi) {
        if constexpr (kBatch) {
          // the next record to apply: the records a trajectory skips (mostly the
          // identity choice of a Pauli slot) go by in a scan of their own, off the
          // loop edge that carries the amplitude registers
#pragma unroll 1
          for (; gi < stg.g1; ++gi) {
            const SwGate& q = p.gates[gi];
            if (((uint64_t)base & q.gmask) != q.gmask) continue;
            if ((q.kind == SK_PAULI || q.kind == SK_PAULIF) && codes[q.b] == 0) continue;
            break;
          }
          if (gi >= stg.g1) break;
        } else {
          if (gi >= stg.g1) break;
          if (((uint64_t)base & p.gates[gi].gmask) != p.gates[gi].gmask) continue;
        }
        const SwGate& g = p.gates[gi];
        const R* m = p.pool + g.moff;
        const uint32_t lmask = g.lmask;
        switch (g.code) {
#define SC_DO_G1(A) g1<R, NR, A>(v, m, l0, off, lmask)
#define SC_DO_X(A)                                                                        \
  smem_permute(v, cur, rbase, tab, [&](int j) {                                           \
    return (((l0 | off[j]) & lmask) == lmask) ? tab.rd[j ^ (1 << (A))] : tab.rd[j];       \
  })
#define SC_DO_D1R(A) d1r<R, NR, A>(v, m)
#define SC_DO_G2(A, B) g2<R, NR, A, B>(v, m)
#define SC_DO_CX(A, B)                                                                    \
  smem_permute(v, cur, rbase, tab, [&](int j) {                                           \
    return (((j >> (B)) & 1) && (l0 & lmask) == lmask) ? tab.rd[j ^ (1 << (A))] : tab.rd[j]; \
  })
#define SC_DO_DPR(A, B) dpr<R, NR, A, B>(v, m)
#define SC_DO_SWAP(A, B)                                                                  \
  smem_permute(v, cur, rbase, tab, [&](int j) {                                           \
    return tab.rd[(((j >> (A)) ^ (j >> (B))) & 1) ? j ^ ((1 << (A)) | (1 << (B))) : j];    \
  })
#define SC_DO_X0(A) smem_permute(v, cur, rbase, tab, [&](int j) { return tab.rd[j ^ (1 << (A))]; })
#define SC_DO_CX0(A, B) \
  smem_permute(v, cur, rbase, tab, [&](int j) { return tab.rd[((j >> (B)) & 1) ? j ^ (1 << (A)) : j]; })
#define SC_DO_PAULI(A)                                                   \
  if constexpr (kBatch) {                                                \
    pauli_slots<R, NR, A>(v, (uint32_t)codes[g.b], cur, rbase, tab);     \
  }
#define SC_DO_XF(A) \
  xfold<NR, A>(sidx, (l0 & lmask) == lmask ? (uint32_t)tab.xoff[A] : 0u)
#define SC_DO_CXF(A, B) \
  cxfold<NR, A, B>(sidx, (l0 & lmask) == lmask ? (uint32_t)tab.xoff[A] : 0u)
          SC_CASES_1(SK_X0, SC_DO_X0)
          SC_CASES_2(SK_CX0, SC_DO_CX0)
          SC_CASES_1(SK_XF, SC_DO_XF)
          SC_CASES_2(SK_CXF, SC_DO_CXF)
#undef SC_DO_XF
#undef SC_DO_CXF
          SC_CASES_1(SK_PAULI, SC_DO_PAULI)
#define SC_DO_TMAT(A)                                                                     \
  if constexpr (kBatch) {                                                                 \
    g1<R, NR, A>(v, p.tmats + ((uint64_t)g.b * (uint64_t)p.batch + (t >> p.tiles_log2)) * 8, \
                 l0, off, 0u);                                                            \
  }
          SC_CASES_1(SK_TMAT, SC_DO_TMAT)
#undef SC_DO_TMAT
          case SK_PAULIF << 4:
            if constexpr (kBatch) {
              pauli_frame_slots<R, NR>(v, m + 3 * ((uint32_t)codes[g.b] - 1u), cur, rbase, tab);
            }
            break;
#undef SC_DO_X0
#undef SC_DO_CX0
#undef SC_DO_PAULI
          SC_CASES_1(SK_G1, SC_DO_G1)
          SC_CASES_1(SK_X, SC_DO_X)
          SC_CASES_1(SK_D1R, SC_DO_D1R)
          SC_CASES_2(SK_G2, SC_DO_G2)
          SC_CASES_2(SK_CX, SC_DO_CX)
          SC_CASES_2(SK_DPR, SC_DO_DPR)
          SC_CASES_2(SK_SWAP, SC_DO_SWAP)
#undef SC_DO_G1
#undef SC_DO_X
#undef SC_DO_D1R
#undef SC_DO_G2
#undef SC_DO_CX
#undef SC_DO_DPR
#undef SC_DO_SWAP
          // commuting 2x2 gates on several register bits, matrices in bit order;
          // one case per bit set, so the gates run as straight-line code
#define SC_G1ALL_CASE(M)                        \
  case (SK_G1ALL << 4) | (M):                   \
    if constexpr (((M) >> NR) == 0) {           \
      g1all<R, NR, (M)>(v, m, l0, off);         \
    }                                           \
    break;
          SC_G1ALL_CASE(1) SC_G1ALL_CASE(2) SC_G1ALL_CASE(3) SC_G1ALL_CASE(4)
          SC_G1ALL_CASE(5) SC_G1ALL_CASE(6) SC_G1ALL_CASE(7) SC_G1ALL_CASE(8)
          SC_G1ALL_CASE(9) SC_G1ALL_CASE(10) SC_G1ALL_CASE(11) SC_G1ALL_CASE(12)
          SC_G1ALL_CASE(13) SC_G1ALL_CASE(14) SC_G1ALL_CASE(15)
#undef SC_G1ALL_CASE
#define SC_G1ALLQ_CASE(M)                                   \
  case (SK_G1ALLQ << 4) | (M):                              \
    if constexpr (((M) >> NR) == 0) {                       \
      if (g.b && !folded_x) {                               \
        const int xb = g.b & (NV - 1);                      \
        smem_permute(v, cur, rbase, tab, [&](int j) { return tab.rd[j ^ xb]; }); \
      }                                                     \
      g1allq<R, NR, (M)>(v, m);                             \
    }                                                       \
    break;
          SC_G1ALLQ_CASE(1) SC_G1ALLQ_CASE(2) SC_G1ALLQ_CASE(3) SC_G1ALLQ_CASE(4)
          SC_G1ALLQ_CASE(5) SC_G1ALLQ_CASE(6) SC_G1ALLQ_CASE(7) SC_G1ALLQ_CASE(8)
          SC_G1ALLQ_CASE(9) SC_G1ALLQ_CASE(10) SC_G1ALLQ_CASE(11) SC_G1ALLQ_CASE(12)
          SC_G1ALLQ_CASE(13) SC_G1ALLQ_CASE(14) SC_G1ALLQ_CASE(15)
#undef SC_G1ALLQ_CASE
          case SK_DTAB << 4:
            dtab<R, NR>(v, m);
            break;
          case SK_D1 << 4:
            diag1_any<R, NR>(v, m, g.a, l0, off, lmask, base);
            break;
          case SK_DP << 4:
            diagp_any<R, NR>(v, m, g.a, g.b, l0, off, base);
            break;
          case SK_D2 << 4:
            diag2_any<R, NR>(v, m, g.a, g.b, l0, off, base);
            break;
          default: break;
        }
      }
    }
    A* __restrict__ dst = item_state(t) + base;
    if (p.has_scale) {
#pragma unroll
      for (int j = 0; j < NV; ++j) v[j] = cmul(p.scale_re, p.scale_im, v[j]);
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) dst[gt_last | p.glast[j]] = v[j];
  }
  if constexpr (kTma) {
    // a thread that stopped waiting may leave tile copies in flight: thread 0 waits
    // (bounded) for the ones it issued before the CTA's shared memory is released
    if (tid == 0 && timed_out) {
      for (uint32_t k = issued >= 2 ? issued - 2 : 0; k < issued; ++k)
        mbar_wait_bounded(&bars[k & 1u], (k >> 1) & 1u, kWaitLimitCycles);
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint reverse pass, fused (addition; the reference has no gradient API).
// The plan holds the inverse gates in reverse order with a probe record before
// each parametrised gate.  One launch carries both states (psi and lambda)
// through the sweep tile by tile: every gate record is applied to both, and a
// probe adds Im sum conj(lambda_i) (P psi)_i over the tile to its gradient slot
// (P the gate's Pauli generator on a register bit).  Probe sums go warp ->
// shared slot per warp -> per-CTA partial, and are added up in a fixed order.
// ---------------------------------------------------------------------------

// Records of the adjoint plan outside the lite set (kLite below): register
// permutations (X, CNOT, SWAP) not folded into a stage's read, 2-qubit diagonals,
// grouped 1-qubit matrices, diagonal tables, diagonals whose bits lie outside the
// registers.
template <typename R, int NR>
__device__ __forceinline__ void apply_record_pair_rest(typename Amp<R>::type (&v)[1 << NR],
                                                       typename Amp<R>::type (&w)[1 << NR],
                                                       const SwGate& g, const R* m, uint32_t l0,
                                                       const RegOff<NR>& off, uint32_t base,
                                                       typename Amp<R>::type* bp,
                                                       typename Amp<R>::type* bl, uint32_t rbase,
                                                       const SwStageTab& tab) {
  const uint32_t lmask = g.lmask;
  // register permutations go through the thread's own slots of both tile buffers
  auto perm2 = [&](auto&& src_rd) {
    smem_permute(v, bp, rbase, tab, src_rd);
    smem_permute(w, bl, rbase, tab, src_rd);
  };
  switch (g.code) {
#define SC_DO_X(A)                                                                          \
  perm2([&](int j) {                                                                        \
    return (((l0 | off[j]) & lmask) == lmask) ? tab.rd[j ^ (1 << (A))] : tab.rd[j];         \
  })
#define SC_DO_CX(A, B)                                                                      \
  perm2([&](int j) {                                                                        \
    return (((j >> (B)) & 1) && (l0 & lmask) == lmask) ? tab.rd[j ^ (1 << (A))] : tab.rd[j]; \
  })
#define SC_DO_X0(A) perm2([&](int j) { return tab.rd[j ^ (1 << (A))]; })
#define SC_DO_CX0(A, B) perm2([&](int j) { return tab.rd[((j >> (B)) & 1) ? j ^ (1 << (A)) : j]; })
    SC_CASES_1(SK_X, SC_DO_X)
    SC_CASES_2(SK_CX, SC_DO_CX)
    SC_CASES_1(SK_X0, SC_DO_X0)
    SC_CASES_2(SK_CX0, SC_DO_CX0)
#undef SC_DO_X
#undef SC_DO_CX
#undef SC_DO_X0
#undef SC_DO_CX0
#define SC_DO_DPR(A, B) dpr<R, NR, A, B>(v, m), dpr<R, NR, A, B>(w, m)
#define SC_DO_SWAP(A, B)                                                                    \
  perm2([&](int j) {                                                                        \
    return tab.rd[(((j >> (A)) ^ (j >> (B))) & 1) ? j ^ ((1 << (A)) | (1 << (B))) : j];     \
  })
    SC_CASES_2(SK_DPR, SC_DO_DPR)
    SC_CASES_2(SK_SWAP, SC_DO_SWAP)
#undef SC_DO_DPR
#undef SC_DO_SWAP
#define SC_G1ALL_CASE(M)                        \
  case (SK_G1ALL << 4) | (M):                   \
    if constexpr (((M) >> NR) == 0) {           \
      g1all<R, NR, (M)>(v, m, l0, off);         \
      g1all<R, NR, (M)>(w, m, l0, off);         \
    }                                           \
    break;
    SC_G1ALL_CASE(1) SC_G1ALL_CASE(2) SC_G1ALL_CASE(3) SC_G1ALL_CASE(4)
    SC_G1ALL_CASE(5) SC_G1ALL_CASE(6) SC_G1ALL_CASE(7) SC_G1ALL_CASE(8)
    SC_G1ALL_CASE(9) SC_G1ALL_CASE(10) SC_G1ALL_CASE(11) SC_G1ALL_CASE(12)
    SC_G1ALL_CASE(13) SC_G1ALL_CASE(14) SC_G1ALL_CASE(15)
#undef SC_G1ALL_CASE
    case SK_DTAB << 4:
      dtab<R, NR>(v, m);
      dtab<R, NR>(w, m);
      break;
    case SK_D1 << 4:
      diag1_any<R, NR>(v, m, g.a, l0, off, lmask, base);
      diag1_any<R, NR>(w, m, g.a, l0, off, lmask, base);
      break;
    case SK_DP << 4:
      diagp_any<R, NR>(v, m, g.a, g.b, l0, off, base);
      diagp_any<R, NR>(w, m, g.a, g.b, l0, off, base);
      break;
    case SK_D2 << 4:
      diag2_any<R, NR>(v, m, g.a, g.b, l0, off, base);
      diag2_any<R, NR>(w, m, g.a, g.b, l0, off, base);
      break;
    default: break;
  }
}

// A record of the adjoint plan applied to both states in one dispatch: one join of
// the register state per record, not two.  kLite: only the records of phase-free
// rotation plans once their register permutations are folded into the stages'
// reads (lifted rotations, half diagonals, 1-qubit matrices, probes).  A case that
// permutes the registers at run time, even one that never runs, makes the record
// loop move the amplitude registers at every record's join (measured: about half
// the instructions of the 26-qubit HEA reverse sweep); the host picks the lite
// kernel when every record the sweep executes is of those kinds.
template <typename R, int NR, bool kLite>
__device__ __forceinline__ void apply_record_pair(typename Amp<R>::type (&v)[1 << NR],
                                                  typename Amp<R>::type (&w)[1 << NR],
                                                  const SwGate& g, const R* m, uint32_t l0,
                                                  const RegOff<NR>& off, uint32_t base,
                                                  typename Amp<R>::type* bp,
                                                  typename Amp<R>::type* bl, uint32_t rbase,
                                                  const SwStageTab& tab) {
  const uint32_t lmask = g.lmask;
  switch (g.code) {
#define SC_DO_G1(A) g1<R, NR, A>(v, m, l0, off, lmask), g1<R, NR, A>(w, m, l0, off, lmask)
#define SC_DO_D1R(A) d1r<R, NR, A>(v, m), d1r<R, NR, A>(w, m)
#define SC_DO_D1H(A) d1h<R, NR, A>(v, m), d1h<R, NR, A>(w, m)
    SC_CASES_1(SK_D1H, SC_DO_D1H)
    SC_CASES_1(SK_G1, SC_DO_G1)
    SC_CASES_1(SK_D1R, SC_DO_D1R)
#undef SC_DO_D1H
#undef SC_DO_G1
#undef SC_DO_D1R
#define SC_ROTL_CASE(M)                         \
  case (SK_ROTL << 4) | (M):                    \
    if constexpr (((M) >> NR) == 0) {           \
      rotl<R, NR, (M)>(v, m);                   \
      rotl<R, NR, (M)>(w, m);                   \
    }                                           \
    break;
    SC_ROTL_CASE(1) SC_ROTL_CASE(2) SC_ROTL_CASE(3) SC_ROTL_CASE(4)
    SC_ROTL_CASE(5) SC_ROTL_CASE(6) SC_ROTL_CASE(7)
#undef SC_ROTL_CASE
    default:
      if constexpr (!kLite) apply_record_pair_rest<R, NR>(v, w, g, m, l0, off, base, bp, bl, rbase, tab);
      break;
  }
}

// the record kinds apply_record_pair<..., kLite = true> handles
inline bool adjoint_lite_kind(int32_t k) {
  return k == SK_ROTL || k == SK_D1H || k == SK_G1 || k == SK_D1R || k == SK_PROBE;
}

// Im sum_j conj(w_j) (P v)_j over the thread's registers, P the Pauli PAULI_
// (1 = X, 2 = Y = iXZ, 3 = Z) on register bit A_ (the planner puts a probed
// qubit in the registers)
template <typename R, int NR, int A_, int PAULI_>
__device__ __forceinline__ double probe_sum(const typename Amp<R>::type (&v)[1 << NR],
                                            const typename Amp<R>::type (&w)[1 << NR]) {
  // two partial sums (even and odd registers): half the dependent FP64 chain
  double s[2] = {0.0, 0.0};
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    const int src = PAULI_ == 3 ? j : j ^ (1 << A_);  // X and Y move the partner in
    double pr = (double)v[src].x, pi = (double)v[src].y;
    if (PAULI_ != 1 && ((src >> A_) & 1)) {  // the Z factor: sign of the source bit
      pr = -pr;
      pi = -pi;
    }
    if (PAULI_ == 2) {  // Y = i X Z
      const double t = pr;
      pr = -pi;
      pi = t;
    }
    s[j & 1] += (double)w[j].x * pi - (double)w[j].y * pr;
  }
  return s[0] + s[1];
}

// THREADS threads per tile, MINB CTAs per SM (their register cap: 65536 / (THREADS x
// MINB)).  While a tile computes, each thread asks L2 for its amplitudes of the
// CTA's next tile (`prefetch.global.L2`: no registers, no wait).
template <typename R, int NR, int THREADS, int MINB, bool kLite>
__global__ void __launch_bounds__(THREADS, MINB)
    k_adjoint_sweep(typename Amp<R>::type* __restrict__ psi, typename Amp<R>::type* __restrict__ lam,
                    const __grid_constant__ SweepParams<R> p, double* __restrict__ partial,
                    int n_probes) {
  using A = typename Amp<R>::type;
  constexpr int NV = 1 << NR;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t tile_amps = 1u << p.T;
  A* const bp = reinterpret_cast<A*>(smem_raw);
  A* const bl = bp + tile_amps;
  double* const acc = reinterpret_cast<double*>(bl + tile_amps);  // [probe][warp]
  const uint32_t tid = threadIdx.x;
  const uint32_t nwarps = blockDim.x >> 5;  // blockDim.x is a multiple of 32 (host check)
  const uint32_t warp = tid >> 5;
  for (uint32_t k = tid; k < (uint32_t)n_probes * nwarps; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();
  const int ns = p.n_stages;
  const uint32_t l0_first = stage_l0<NR>(tid, p.stages[0]);
  const uint32_t l0_last = stage_l0<NR>(tid, p.stages[ns - 1]);
  const uint32_t gt_first = spread32(l0_first, p);
  const uint32_t gt_last = spread_out32(l0_last, p);
  for (uint32_t t = blockIdx.x; t < (uint32_t)p.tiles; t += gridDim.x) {
    // a permutation record of the full kernel works in the thread's own slots of the
    // current stage's layout: every thread is past the last tile's final reads first
    if constexpr (!kLite) __syncthreads();
    const uint32_t base = tile_base(t, p);
    // the read flip of a stage's conditional entry folds (tab.rf_off, or the first
    // stage's global offsets rf_goff0), for the thread's stage base
    auto entry_flip = [&](const SwStageTab& tab, uint32_t lbase, bool global) -> uint32_t {
      uint32_t f = 0;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (tab.rf_g[k] < 0) continue;
        const SwGate& q = p.gates[tab.rf_g[k]];
        if (((uint64_t)base & q.gmask) == q.gmask && (lbase & q.lmask) == q.lmask)
          f ^= global ? p.rf_goff0[k] : (uint32_t)tab.rf_off[k];
      }
      return f;
    };
    A v[NV], w[NV];
    {
      // the flip moves register-position bits only (disjoint from base and gt_first)
      const uint32_t gfl = entry_flip(p.tabs[0], l0_first, true);
#pragma unroll
      for (int j = 0; j < NV; ++j) {
        v[j] = psi[base | gt_first | (p.gread0[j] ^ gfl)];
        w[j] = lam[base | gt_first | (p.gread0[j] ^ gfl)];
      }
    }
    if (t + gridDim.x < (uint32_t)p.tiles) {
      const uint32_t nb = tile_base(t + gridDim.x, p);
#pragma unroll
      for (int j = 0; j < NV; ++j) {
        prefetch_l2(psi + (nb | gt_first | p.gfirst[j]));
        prefetch_l2(lam + (nb | gt_first | p.gfirst[j]));
      }
    }
    // the thread's read base in the current stage (the first stage: its linear slots)
    uint32_t rbase = l0_first;
    uint32_t l0 = l0_first, psw0 = 0;
    RegOff<NR> off;
#pragma unroll 1
    for (int s = 0; s < ns; ++s) {
      const SwStage& stg = p.stages[s];
      const SwStageTab& tab = p.tabs[s];
      const uint32_t nl0 = (s == 0) ? l0_first : stage_l0<NR>(tid, stg);
      const uint32_t sw0 = swz<R>(nl0);
      if (s > 0) {
        __syncthreads();  // readers of the buffers are done
        // the previous stage's exit slots (its folded permutation applied)
        const SwStageTab& ptab = p.tabs[s - 1];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          bp[psw0 ^ ptab.wsoff[j]] = v[j];
          bl[psw0 ^ ptab.wsoff[j]] = w[j];
        }
        __syncthreads();
        rbase = sw0 ^ entry_flip(tab, nl0, false);
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          v[j] = bp[rbase ^ tab.rd[j]];
          w[j] = bl[rbase ^ tab.rd[j]];
        }
      }
      psw0 = sw0;
      l0 = nl0;
#pragma unroll
      for (int k = 0; k < NR; ++k) off.rb[k] = 1u << stg.R[k];
#pragma unroll 1
      for (int gi = stg.g0; gi < stg.g1; ++gi) {
        const SwGate& g = p.gates[gi];
        if (((uint64_t)base & g.gmask) != g.gmask) continue;
        if (g.kind == SK_PROBE) {
          // Up to four consecutive probes (one point of the plan: the probes of a
          // run of rotations) are summed and then reduced over the warp together,
          // their shuffle trees interleaved instead of one after another.
          auto probe = [&](const SwGate& q) -> double {
            double ps = 0.0;
            switch (q.code & 15) {
#define SC_PROBE_CASE(A, P)                      \
  case ((A) << 2) | (P):                         \
    if constexpr ((A) < NR) ps = probe_sum<R, NR, (A), (P)>(v, w); \
    break;
              SC_PROBE_CASE(0, 1) SC_PROBE_CASE(0, 2) SC_PROBE_CASE(0, 3)
              SC_PROBE_CASE(1, 1) SC_PROBE_CASE(1, 2) SC_PROBE_CASE(1, 3)
              SC_PROBE_CASE(2, 1) SC_PROBE_CASE(2, 2) SC_PROBE_CASE(2, 3)
              SC_PROBE_CASE(3, 1) SC_PROBE_CASE(3, 2) SC_PROBE_CASE(3, 3)
#undef SC_PROBE_CASE
              default: break;
            }
            return ps;
          };
          // the next record joins the group when it is a probe (probes carry no
          // global controls)
          auto next_probe = [&]() {
            return gi + 1 < stg.g1 && p.gates[gi + 1].kind == SK_PROBE && p.gates[gi + 1].gmask == 0;
          };
          double p0 = probe(g), p1 = 0.0, p2 = 0.0, p3 = 0.0;
          const uint32_t b0 = (uint32_t)g.b;  // b: local probe index
          uint32_t b1 = 0, b2 = 0, b3 = 0;
          int np = 1;
          if (next_probe()) {
            ++gi;
            p1 = probe(p.gates[gi]);
            b1 = (uint32_t)p.gates[gi].b;
            np = 2;
            if (next_probe()) {
              ++gi;
              p2 = probe(p.gates[gi]);
              b2 = (uint32_t)p.gates[gi].b;
              np = 3;
              if (next_probe()) {
                ++gi;
                p3 = probe(p.gates[gi]);
                b3 = (uint32_t)p.gates[gi].b;
                np = 4;
              }
            }
          }
          if (np <= 2) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              p0 += __shfl_xor_sync(0xffffffffu, p0, o);
              p1 += __shfl_xor_sync(0xffffffffu, p1, o);
            }
          } else {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              p0 += __shfl_xor_sync(0xffffffffu, p0, o);
              p1 += __shfl_xor_sync(0xffffffffu, p1, o);
              p2 += __shfl_xor_sync(0xffffffffu, p2, o);
              p3 += __shfl_xor_sync(0xffffffffu, p3, o);
            }
          }
          if ((tid & 31u) == 0) {
            acc[b0 * nwarps + warp] += p0;
            if (np > 1) acc[b1 * nwarps + warp] += p1;
            if (np > 2) acc[b2 * nwarps + warp] += p2;
            if (np > 3) acc[b3 * nwarps + warp] += p3;
          }
          continue;
        }
        apply_record_pair<R, NR, kLite>(v, w, g, p.pool + g.moff, l0, off, base, bp, bl, rbase, tab);
      }
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      psi[base | gt_last | p.glast[j]] = v[j];
      lam[base | gt_last | p.glast[j]] = w[j];
    }
  }
  __syncthreads();
  for (uint32_t k = tid; k < (uint32_t)n_probes; k += blockDim.x) {
    double sum = 0.0;
    for (uint32_t q = 0; q < nwarps; ++q) sum += acc[k * nwarps + q];
    partial[(size_t)blockIdx.x * (size_t)n_probes + k] = sum;
  }
}

// grad[slot[k]] += sum over CTAs of partial[cta][k], CTAs in order (one thread per probe)
struct ProbeSlots {
  int32_t slot[kSweepMaxGates];
};

__global__ void k_probe_reduce(const double* __restrict__ partial, int ctas, int n_probes,
                               const __grid_constant__ ProbeSlots slots, double* __restrict__ grad) {
  const int k = (int)threadIdx.x;
  if (k >= n_probes) return;
  double sum = 0.0;
  for (int b = 0; b < ctas; ++b) sum += partial[(size_t)b * (size_t)n_probes + k];
  grad[slots.slot[k]] += sum;
}

struct LaunchCache {
  std::mutex mu;
  bool attr_set[2][SW_MAX_NR + 1][2][2] = {};
};
LaunchCache g_cache;

// cuTensorMapEncodeTiled, looked up once through the runtime (no link-time
// dependency on the driver library)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    if (const char* v = getenv("STATECRAFT_B200_TMA"))
      if (atoi(v) == 0) return;  // tensor copies off: every sweep takes the cp.async path
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

// The state (or the batch of states) as the copy engine sees it, so that each tile
// of a sweep is one box (layout in sc_sweep.h): dims, byte strides and box of each
// dim, innermost first, with the coordinate rules stored into p.  False when the
// tile is not a box of at most kTileTensorMaxRank dims in its linear order.
struct TileTensor {
  int rank = 0;
  uint64_t dims[kTileTensorMaxRank];     // in 8-byte elements for dim 0, else in steps
  uint64_t strides[kTileTensorMaxRank];  // bytes per step (dim 0: the element)
  uint32_t box[kTileTensorMaxRank];
};

template <typename R>
bool tile_tensor_geometry(SweepParams<R>& p, TileTensor* tt) {
  using A = typename Amp<R>::type;
  p.tm_rank = 0;
  for (int k = 0; k < kTileTensorMaxRank; ++k) {
    p.tm_shift[k] = 0;
    p.tm_mask[k] = 0;
  }
  if (p.relayout || p.L < 1) return false;
  const int n = p.nq;
  // tile bits: 0..L-1 and hq[] ascending, so the box lands in the linear tile order
  uint64_t tile = (1ULL << p.L) - 1ULL;
  for (int k = 0; k < p.h; ++k) {
    if (p.hq[k] < p.L || p.hq[k] >= n || (k > 0 && p.hq[k] <= p.hq[k - 1])) return false;
    tile |= 1ULL << p.hq[k];
  }
  const int e = (int)(sizeof(A) / 8);  // 8-byte elements per amplitude
  int rank = 0, nontile_below = 0;
  for (int b = 0; b < n;) {
    const bool in = ((tile >> b) & 1ULL) != 0;
    int len = 0;
    while (b + len < n && (((tile >> (b + len)) & 1ULL) != 0) == in) ++len;
    // a box dim holds at most 256 elements: long tile runs take several dims
    for (int start = b, rem = len; rem > 0;) {
      const int cap = in ? (start == 0 ? (e == 2 ? 7 : 8) : 8) : 32;
      const int w = std::min(rem, cap);
      if (rank >= kTileTensorMaxRank) return false;
      tt->dims[rank] = (uint64_t)(start == 0 ? e : 1) << w;
      tt->box[rank] = in ? (uint32_t)tt->dims[rank] : 1u;
      tt->strides[rank] = start == 0 ? 8u : (uint64_t)sizeof(A) << start;
      p.tm_shift[rank] = in ? 0 : nontile_below;
      p.tm_mask[rank] = in ? 0u : (uint32_t)((1ULL << w) - 1ULL);
      if (!in) nontile_below += w;
      ++rank;
      start += w;
      rem -= w;
    }
    b += len;
  }
  if (p.batch > 1) {  // the state index of a batch
    if (rank >= kTileTensorMaxRank) return false;
    tt->dims[rank] = (uint64_t)p.batch;
    tt->box[rank] = 1u;
    tt->strides[rank] = (uint64_t)sizeof(A) << n;
    p.tm_shift[rank] = p.tiles_log2;
    p.tm_mask[rank] = 0xffffffffu;
    ++rank;
  }
  tt->rank = rank;
  return true;
}

// Fills p.tmap for the state at `state` and sets p.tm_rank; false (tm_rank = 0) when
// the sweep has no box form or the encoder is unavailable or refuses it.
template <typename R>
bool make_tile_tensor(void* state, SweepParams<R>& p) {
  TileTensor tt;
  EncodeTiledFn encode = encode_tiled_fn();
  if (!encode || !tile_tensor_geometry(p, &tt)) {
    p.tm_rank = 0;
    return false;
  }
  cuuint64_t dims[kTileTensorMaxRank], strides[kTileTensorMaxRank];
  cuuint32_t box[kTileTensorMaxRank], estr[kTileTensorMaxRank];
  for (int k = 0; k < tt.rank; ++k) {
    dims[k] = tt.dims[k];
    strides[k] = tt.strides[k];
    box[k] = tt.box[k];
    estr[k] = 1;
  }
  static_assert(sizeof(p.tmap) == sizeof(CUtensorMap), "tensor map storage");
  const CUresult r = encode(reinterpret_cast<CUtensorMap*>(p.tmap), CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                            (cuuint32_t)tt.rank, state, dims, strides + 1, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    p.tm_rank = 0;
    return false;
  }
  p.tm_rank = tt.rank;
  return true;
}

// Host check of the box geometry: for every work item and every tile position, the
// global amplitude the box copies to that position of the tile buffer (copy-engine
// addressing: shared offset = box-linear index, global offset = sum over dims of
// (coordinate + index) * stride) is the one the sweep's tile enumeration assigns
// to it.  stats[0] += sweeps with a box form, stats[1] += work items checked.
template <typename R>
bool check_tile_tensor(SweepParams<R>& p, int64_t* stats) {
  using A = typename Amp<R>::type;
  TileTensor tt;
  if (!tile_tensor_geometry(p, &tt)) return true;  // cp.async path: nothing to check
  const int e = (int)(sizeof(A) / 8);
  uint64_t box_elems = 1;
  for (int k = 0; k < tt.rank; ++k) box_elems *= tt.box[k];
  if (box_elems != (uint64_t)e << p.T) return false;  // the tile is exactly one box
  if (tt.dims[0] != tt.box[0] || (tt.box[0] * 8u) % 16u != 0) return false;
  const uint64_t items = (uint64_t)p.tiles * (uint64_t)p.batch;
  const uint64_t step = items > 4096 ? items / 4096 : 1;  // a spread of items
  for (uint64_t it = 0; it < items; it += step) {
    int32_t c[kTileTensorMaxRank];
    for (int k = 0; k < tt.rank; ++k) {
      c[k] = (int32_t)((it >> p.tm_shift[k]) & p.tm_mask[k]);
      if ((uint64_t)c[k] + tt.box[k] > tt.dims[k]) return false;
    }
    const uint64_t tile = it & ((uint64_t)p.tiles - 1ULL);
    const uint64_t st = it >> p.tiles_log2;
    const uint64_t base = tile_base((uint32_t)tile, p);
    for (uint64_t sm = 0; sm < box_elems; sm += (uint64_t)e) {
      // decompose the shared offset into per-dim box indices, dim 0 fastest
      uint64_t rest = sm, byte = 0;
      for (int k = 0; k < tt.rank; ++k) {
        const uint64_t idx = rest % tt.box[k];
        rest /= tt.box[k];
        byte += ((uint64_t)c[k] + idx) * tt.strides[k];
      }
      const uint64_t want = (st << p.nq) | base | host_spread_t(sm / (uint64_t)e, p);
      if (byte != want * sizeof(A)) return false;
    }
    ++stats[1];
  }
  ++stats[0];
  return true;
}

template <typename R, int NR, bool kTma, bool kBatch>
cudaError_t launch_nr(void* state, const SweepParams<R>& p, int* err, int sm_count,
                      cudaStream_t s) {
  using A = typename Amp<R>::type;
  auto kern = k_sweep<R, NR, kTma, kBatch>;
  const int di = std::is_same<R, float>::value ? 1 : 0;
  {
    std::lock_guard<std::mutex> lk(g_cache.mu);
    if (!g_cache.attr_set[di][NR][kTma][kBatch]) {
      cudaError_t e =
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return e;
      g_cache.attr_set[di][NR][kTma][kBatch] = true;
    }
  }
  const int threads = 1 << (p.T - NR);
  if (threads > sweep_max_threads<R, NR>()) return cudaErrorInvalidConfiguration;
  const size_t smem = sweep_smem_bytes<R>(p.T);
  if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  per_sm = std::max(per_sm, 1);
  const int64_t grid = std::min<int64_t>(p.tiles * p.batch, (int64_t)sm_count * per_sm);
  kern<<<(unsigned)grid, threads, smem, s>>>(static_cast<A*>(state), p, err);
  return cudaGetLastError();
}

template <typename R, int NR>
cudaError_t launch_pick(void* state, SweepParams<R>& p, int* err, int sm_count, cudaStream_t s) {
  const bool batch = p.batch > 1 || p.n_local_slots > 0 || p.tmats != nullptr;
  p.stall_first = 0;
  if (const char* v = getenv("STATECRAFT_B200_TEST_STALL_CYCLES")) p.stall_first = atoi(v);
  if (make_tile_tensor<R>(state, p))
    return batch ? launch_nr<R, NR, true, true>(state, p, err, sm_count, s)
                 : launch_nr<R, NR, true, false>(state, p, err, sm_count, s);
  return batch ? launch_nr<R, NR, false, true>(state, p, err, sm_count, s)
               : launch_nr<R, NR, false, false>(state, p, err, sm_count, s);
}

template <typename R>
cudaError_t launch_t(void* state, SweepParams<R>& p, int* err, int sm_count, cudaStream_t s) {
  switch (p.nr) {
    case 1: return launch_pick<R, 1>(state, p, err, sm_count, s);
    case 2: return launch_pick<R, 2>(state, p, err, sm_count, s);
    case 3: return launch_pick<R, 3>(state, p, err, sm_count, s);
    case 4: return launch_pick<R, 4>(state, p, err, sm_count, s);
    default: return cudaErrorInvalidValue;
  }
}

uint32_t host_spread(uint32_t x, const SwSweep& sw) {
  uint32_t g = x & ((1u << sw.L) - 1u);
  uint32_t hi = x >> sw.L;
  for (int k = 0; hi; ++k, hi >>= 1)
    if (hi & 1u) g |= 1u << sw.hq[k];
  return g;
}

uint32_t host_spread_out(uint32_t x, const SwSweep& sw) {
  uint32_t g = 0;
  for (int k = 0; x; ++k, x >>= 1)
    if (x & 1u) g |= 1u << sw.outp[k];
  return g;
}

// An exchange swizzle (SwStageTab::rows): slot(i) = i ^ sum_k parity(i & rows[k]) << k.
struct ExchangeSwizzle {
  uint16_t rows[4];
  bool general;
};

uint32_t apply_swizzle(uint32_t i, const ExchangeSwizzle& z, int K) {
  uint32_t lo = 0;
  for (int k = 0; k < K; ++k) lo |= (uint32_t)(__builtin_popcount(i & z.rows[k]) & 1) << k;
  return i ^ lo;
}

// Tile positions of thread-index bits 0..K-1 in a stage: the threads whose accesses
// share one 128-byte shared-memory wavefront differ in exactly these positions.
void wavefront_positions(const SwStage& st, int nr, int K, int* pos) {
  for (int b = 0; b < K; ++b) {
    uint32_t x = 1u << b;
    for (int k = 0; k < nr; ++k) x = insert_zero32(x, st.R[k]);
    pos[b] = __builtin_ctz(x);
  }
}

// The swizzle of one exchange: the slot-bit vectors of the writer's m wavefront
// positions (pw; m = K, or the thread bits of a tile with fewer threads than a
// wavefront) must be linearly independent over GF(2) (distinct bank groups), and so
// must the reader's (pr).  Position p < K contributes the unit vector of bit
// p, position p >= K its column col[p] (bit k of col[p] = bit p of rows[k]).  The
// default columns (col[K + k] = 1 << k) are kept when they serve both sides;
// otherwise the columns of the wavefront positions >= K are searched.
ExchangeSwizzle exchange_swizzle(const int* pw, const int* pr, int m, int K, int T) {
  int col[16] = {0};
  auto set_default = [&]() {
    for (int p = 0; p < 16; ++p) col[p] = (p >= K && p < 2 * K && p < T) ? 1 << (p - K) : 0;
  };
  set_default();
  auto vec = [&](int p) { return p < K ? 1 << p : col[p]; };
  // independence of the vectors of ps whose position is decided (< K, or in `fixed`)
  auto independent = [&](const int* ps, uint32_t fixed) {
    uint32_t span = 1u;  // bit u set: vector u lies in the span
    for (int b = 0; b < m; ++b) {
      if (ps[b] >= K && !((fixed >> ps[b]) & 1u)) continue;
      const int v = vec(ps[b]);
      if ((span >> v) & 1u) return false;
      uint32_t nspan = span;
      for (int u = 0; u < (1 << K); ++u)
        if ((span >> u) & 1u) nspan |= 1u << (u ^ v);
      span = nspan;
    }
    return true;
  };
  ExchangeSwizzle z{};
  const bool fits = K <= 4 && T <= 15;
  bool ok = fits && independent(pw, 0xffffu) && independent(pr, 0xffffu);
  if (!ok && fits) {
    int q[8], nq = 0;
    for (int side = 0; side < 2; ++side)
      for (int b = 0; b < m; ++b) {
        const int p = side ? pr[b] : pw[b];
        bool seen = p < K;
        for (int i = 0; i < nq; ++i) seen = seen || q[i] == p;
        if (!seen) q[nq++] = p;
      }
    // depth-first over the columns of q, pruned on the decided positions
    int choice[8] = {0};
    int i = 0;
    uint32_t fixed = 0;
    long budget = 1L << 16;  // bounds the planning time; the default stays correct
    while (i >= 0 && budget-- > 0) {
      if (i == nq) {
        ok = true;
        break;
      }
      if (++choice[i] >= (1 << K)) {  // exhausted: back up
        choice[i] = 0;
        fixed &= ~(1u << q[i]);
        --i;
        continue;
      }
      col[q[i]] = choice[i];
      fixed |= 1u << q[i];
      if (independent(pw, fixed) && independent(pr, fixed)) ++i;
    }
    z.general = ok;
    if (!ok) set_default();  // the default is correct, only with bank conflicts
  }
  for (int k = 0; k < 4; ++k) {
    z.rows[k] = 0;
    if (k < K)
      for (int p = K; p < T && p < 15; ++p)
        if ((col[p] >> k) & 1) z.rows[k] |= (uint16_t)(1u << p);
  }
  if (z.general) z.rows[0] |= 0x8000u;
  return z;
}

// Copies sweep `k` of `plan` into the kernel-parameter form (sweep-local indices,
// per-stage register tables).
// exchange_swizzles: give each exchange its own conflict-free swizzle (the fused
// sweep kernel); false keeps the fixed swizzle (the adjoint kernel).
template <typename R>
bool fill_params(const Plan& plan, size_t k, SweepParams<R>* p, bool exchange_swizzles = true) {
  const SwSweep& sw = plan.sweeps[k];
  const int ns = sw.s1 - sw.s0;
  if (ns < 1 || ns > kSweepMaxStages || sw.nr > SW_MAX_NR) return false;
  const int g_lo = sweep_first_gate(plan, sw), g_hi = plan.stages[sw.s1 - 1].g1;
  if (g_hi - g_lo > kSweepMaxGates) return false;
  p->tm_rank = 0;
  p->stall_first = 0;
  p->T = sw.T;
  p->L = sw.L;
  p->h = sw.h;
  p->nr = sw.nr;
  p->n_stages = ns;
  p->relayout = sw.relayout;
  p->scale_re = (R)sw.scale_re;
  p->scale_im = (R)sw.scale_im;
  p->has_scale = !(sw.scale_re == 1.0 && sw.scale_im == 0.0);
  p->pad3 = 0;
  p->tiles = sw.tiles;
  p->nq = sw.T + (int32_t)__builtin_ctzll((uint64_t)sw.tiles);
  p->n_slots = 0;
  p->tiles_log2 = (int32_t)__builtin_ctzll((uint64_t)sw.tiles);
  p->pad2 = 0;
  p->batch = 1;
  p->paulis = nullptr;
  p->tmats = nullptr;
  p->n_local_slots = 0;
  for (int q = 0; q < SW_MAX_HIGH; ++q) {
    p->hq[q] = sw.hq[q];
    p->hs[q] = sw.hs[q];
  }
  for (int q = 0; q < 32; ++q) p->outp[q] = (uint8_t)sw.outp[q];
  const int K = Amp<R>::kSwizzleShift;
  const int nv = 1 << sw.nr;
  // the swizzle of the layout each stage reads (stage 0 reads the linear layout)
  std::vector<ExchangeSwizzle> zin(ns);
  {
    const int low[4] = {0, 1, 2, 3};
    const ExchangeSwizzle dflt = exchange_swizzle(low, low, K, K, sw.T);
    for (int s = 0; s < ns; ++s) zin[s] = dflt;
    const int m = std::min(K, sw.T - sw.nr);  // thread bits sharing one wavefront
    if (exchange_swizzles && m > 0) {
      for (int s = 1; s < ns; ++s) {
        int pw[4], pr[4];
        wavefront_positions(plan.stages[sw.s0 + s - 1], sw.nr, m, pw);
        wavefront_positions(plan.stages[sw.s0 + s], sw.nr, m, pr);
        zin[s] = exchange_swizzle(pw, pr, m, K, sw.T);
      }
    }
  }
  for (int s = 0; s < ns; ++s) {
    SwStage st = plan.stages[sw.s0 + s];
    st.g0 -= g_lo;
    st.g1 -= g_lo;
    p->stages[s] = st;
    const ExchangeSwizzle& zout = zin[s + 1 < ns ? s + 1 : s];
    for (int b = 0; b < 4; ++b) {
      p->tabs[s].rows[b] = zin[s].rows[b];
      p->tabs[s].xoff[b] =
          b < sw.nr ? (uint16_t)apply_swizzle(1u << st.R[b], zout, K) : (uint16_t)0;
    }
    uint16_t off[16];
    for (int j = 0; j < 16; ++j) {
      uint32_t o = 0;
      if (j < nv)
        for (int b = 0; b < sw.nr; ++b)
          if (j & (1 << b)) o |= 1u << st.R[b];
      off[j] = (uint16_t)o;
    }
    if (s == 0)
      for (int j = 0; j < 16; ++j) p->off0[j] = off[j];
    // a stage whose only register record is one rotation record (other records being
    // slot folds, which act at the exit) reads its registers with the record's
    // leading X already applied
    int n_rot = 0, n_other = 0, rot_g = -1;
    for (int g = plan.stages[sw.s0 + s].g0; g < plan.stages[sw.s0 + s].g1; ++g) {
      const SwGate& q = plan.gates[g];
      if (q.kind == SK_XF || q.kind == SK_CXF) continue;
      if (q.kind == SK_G1ALLQ && q.lmask == 0 && q.gmask == 0) {
        ++n_rot;
        rot_g = g;
      } else {
        ++n_other;
      }
    }
    SwStageTab& tb = p->tabs[s];
    tb.xm = (int8_t)((n_other == 0 && n_rot == 1) ? (plan.gates[rot_g].b & (nv - 1)) : 0);
    tb.pad = 0;
    // register j reads the amplitude of register sigma(j ^ xm) of the plain read: the
    // stage's entry folds, then the folded leading X of its rotation record
    const StageEntry en = plan.entry.empty() ? StageEntry() : plan.entry[sw.s0 + s];
    for (int j = 0; j < 16; ++j) {
      const int jx = j < nv ? en.rperm[j ^ tb.xm] : j;
      if (jx < 0 || jx >= 16) return false;
      tb.rd[j] = s == 0 ? off[jx] : (uint16_t)apply_swizzle(off[jx], zin[s], K);
    }
    for (int k = 0; k < 2; ++k) {
      tb.rf_g[k] = -1;
      tb.rf_off[k] = 0;
      if (k >= en.n_rf) continue;
      if (en.rf_g[k] < g_lo || en.rf_g[k] >= g_hi || en.rf_d[k] <= 0 || en.rf_d[k] >= nv)
        return false;
      tb.rf_g[k] = (int8_t)(en.rf_g[k] - g_lo);
      tb.rf_off[k] = s == 0 ? off[en.rf_d[k]] : (uint16_t)apply_swizzle(off[en.rf_d[k]], zin[s], K);
    }
    if (s == 0) {
      for (int j = 0; j < 16; ++j)
        p->gread0[j] = host_spread(off[j < nv ? en.rperm[j ^ tb.xm] : j], sw);
      for (int k = 0; k < 2; ++k)
        p->rf_goff0[k] = k < en.n_rf ? host_spread(off[en.rf_d[k]], sw) : 0u;
    }
    for (int j = 0; j < 16; ++j) {
      const int pj = (j < nv) ? st.perm[j] : j;
      if (pj < 0 || pj >= 16) return false;
      tb.wsoff[j] = (uint16_t)apply_swizzle(off[pj], zout, K);
    }
    if (s == ns - 1)
      for (int j = 0; j < 16; ++j) p->lastoff[j] = off[(j < nv) ? st.perm[j] : j];
  }
  // slot folds act on the exchange slots: none may sit in the last stage
  for (int g = plan.stages[sw.s1 - 1].g0; g < plan.stages[sw.s1 - 1].g1; ++g)
    if (plan.gates[g].kind == SK_XF || plan.gates[g].kind == SK_CXF) return false;
  for (int j = 0; j < 16; ++j) {
    p->gfirst[j] = host_spread(p->off0[j], sw);
    p->glast[j] = host_spread_out(p->lastoff[j], sw);
  }
  // the sweep's record data: the pool entries appended while it was planned (records
  // need not reference them in order: the stage peephole moves records)
  const int32_t pool_lo = sw.pool0, pool_hi = sw.pool1;
  for (int g = g_lo; g < g_hi; ++g) {
    SwGate sg = plan.gates[g];
    if (sg.moff < pool_lo || sg.moff > pool_hi) return false;
    sg.moff -= pool_lo;
    if (sg.kind == SK_PAULI || sg.kind == SK_PAULIF) {  // slot -> local index into the staged choices
      if (p->n_local_slots >= kSweepMaxGates) return false;
      p->slot_map[p->n_local_slots] = sg.b;
      sg.b = p->n_local_slots++;
    }
    p->gates[g - g_lo] = sg;
  }
  if (pool_hi < pool_lo || pool_hi - pool_lo > kSweepMaxPool) return false;
  for (int32_t e = pool_lo; e < pool_hi; ++e) p->pool[e - pool_lo] = (R)plan.pool[e];
  p->pool_len = pool_hi - pool_lo;
  return true;
}

}  // namespace

namespace {

template <typename R>
bool check_exchanges_t(const Plan& plan, int64_t* st) {
  const int K = Amp<R>::kSwizzleShift;
  // the kernel's slot map (stage_swz), restated on the host
  auto slot_of = [&](uint32_t i, const SwStageTab& t) {
    if (!(t.rows[0] & 0x8000u)) return i ^ ((i >> K) & ((1u << K) - 1u));
    uint32_t lo = 0;
    for (int k = 0; k < K; ++k) lo |= (uint32_t)(__builtin_popcount(i & t.rows[k]) & 1) << k;
    return i ^ lo;
  };
  auto l0_of = [](uint32_t tid, const SwStage& s, int nr) {
    for (int k = 0; k < nr; ++k) tid = insert_zero32(tid, s.R[k]);
    return tid;
  };
  std::unique_ptr<SweepParams<R>> pp(new SweepParams<R>());
  SweepParams<R>& p = *pp;
  for (size_t k = 0; k < plan.sweeps.size(); ++k) {
    if (!fill_params(plan, k, &p)) return false;
    const int T = p.T, nr = p.nr, NV = 1 << nr, threads = 1 << (T - nr);
    for (int s = 1; s < p.n_stages; ++s) {
      ++st[0];
      if (p.tabs[s].rows[0] & 0x8000u) ++st[1];
      std::vector<int64_t> wslot((size_t)1 << T, -1), rslot((size_t)1 << T, -1);
      const SwStage& sw = p.stages[s - 1];
      const SwStage& sr = p.stages[s];
      auto off_of = [&](const SwStage& g, int j) {
        uint32_t o = 0;
        for (int b = 0; b < nr; ++b)
          if (j & (1 << b)) o |= 1u << g.R[b];
        return o;
      };
      for (int tid = 0; tid < threads; ++tid) {
        const uint32_t lw = l0_of(tid, sw, nr), lr = l0_of(tid, sr, nr);
        const uint32_t bw = slot_of(lw, p.tabs[s]), br = slot_of(lr, p.tabs[s]);
        for (int j = 0; j < NV; ++j) {
          const uint32_t a = bw ^ p.tabs[s - 1].wsoff[j];  // register j leaves as perm[j]
          const uint32_t b = br ^ p.tabs[s].rd[j];
          if (a >= (1u << T) || b >= (1u << T) || wslot[a] >= 0 || rslot[b] >= 0) return false;
          wslot[a] = lw | off_of(sw, sw.perm[j]);
          // register j takes the amplitude of register sigma(j ^ xm) (the stage's
          // entry folds and the folded leading X)
          const int jr = plan.entry.empty() ? (j ^ p.tabs[s].xm)
                                            : plan.entry[plan.sweeps[k].s0 + s].rperm[j ^ p.tabs[s].xm];
          rslot[b] = lr | off_of(sr, jr);
        }
        for (int a = 0; a < nr; ++a)
          if (p.tabs[s - 1].xoff[a] != slot_of(1u << sw.R[a], p.tabs[s])) return false;
      }
      if (wslot != rslot) return false;
      // wavefronts: 2^K consecutive threads (all of a smaller tile), one register
      // index, each side
      const int group = std::min(1 << K, threads);
      for (int side = 0; side < 2; ++side)
        for (int t0 = 0; t0 < threads; t0 += group)
          for (int j = 0; j < NV; ++j) {
            uint32_t seen = 0;
            int n = 0;
            for (int t = t0; t < t0 + group; ++t, ++n) {
              const uint32_t a = side == 0
                  ? slot_of(l0_of(t, sw, nr), p.tabs[s]) ^ p.tabs[s - 1].wsoff[j]
                  : slot_of(l0_of(t, sr, nr), p.tabs[s]) ^ p.tabs[s].rd[j];
              seen |= 1u << (a & ((1u << K) - 1u));
            }
            ++st[2];
            if (__builtin_popcount(seen) < n) ++st[3];
          }
    }
    // the linear layout of the tile buffer: the first stage's read (where whole-tile
    // copies and per-thread copies land).  Counted where the planner can put the first
    // stage's registers on high positions (h >= NR) and a wavefront's threads fill it;
    // elsewhere registers sit on low positions, where some conflict is unavoidable
    const int group = 1 << K;
    const bool counted = threads >= group && p.h >= nr;
    for (int side = 0; side < (counted ? 1 : 0); ++side) {
      const SwStage& sg = p.stages[0];
      for (int t0 = 0; t0 < threads; t0 += group)
        for (int j = 0; j < NV; ++j) {
          uint32_t seen = 0;
          int n = 0;
          for (int t = t0; t < t0 + group; ++t, ++n) {
            const uint32_t a = l0_of(t, sg, nr) ^ p.tabs[0].rd[j];
            seen |= 1u << (a & ((1u << K) - 1u));
          }
          ++st[2];
          if (__builtin_popcount(seen) < n) ++st[3];
        }
    }
  }
  return true;
}

}  // namespace

namespace {

template <typename R>
bool check_tile_tensors_t(const Plan& plan, int64_t batch, int64_t* stats) {
  std::unique_ptr<SweepParams<R>> pp(new SweepParams<R>());
  for (size_t k = 0; k < plan.sweeps.size(); ++k) {
    if (!fill_params(plan, k, pp.get())) return false;
    pp->batch = batch;
    if (!check_tile_tensor(*pp, stats)) return false;
  }
  return true;
}

}  // namespace

bool check_tile_tensors(const Plan& plan, int dtype, int64_t batch, int64_t* stats) {
  stats[0] = stats[1] = 0;
  return dtype == SC_C64 ? check_tile_tensors_t<float>(plan, batch, stats)
                         : check_tile_tensors_t<double>(plan, batch, stats);
}

bool check_exchange_tables(const Plan& plan, int dtype, int64_t* stats) {
  for (int i = 0; i < 4; ++i) stats[i] = 0;
  return dtype == SC_C64 ? check_exchanges_t<float>(plan, stats)
                         : check_exchanges_t<double>(plan, stats);
}

cudaError_t launch_sweep(int dtype, void* state, const Plan& plan, size_t k, int* err,
                         int sm_count, cudaStream_t s) {
  if (dtype == SC_C64) {
    SweepParams<float> p;
    if (!fill_params(plan, k, &p)) return cudaErrorInvalidValue;
    return launch_t<float>(state, p, err, sm_count, s);
  }
  SweepParams<double> p;
  if (!fill_params(plan, k, &p)) return cudaErrorInvalidValue;
  return launch_t<double>(state, p, err, sm_count, s);
}

cudaError_t launch_sweep_batch(int dtype, void* states, int n, int64_t batch, const Plan& plan,
                               size_t k, const uint8_t* paulis, int n_slots, const void* tmats,
                               int* err, int sm_count, cudaStream_t s) {
  if (batch < 1 || ((uint64_t)plan.sweeps[k].tiles * (uint64_t)batch) > 0xffffffffull)
    return cudaErrorInvalidValue;
  auto fill = [&](auto* p) {
    if (!fill_params(plan, k, p)) return false;
    if (p->nq != n) return false;
    p->batch = batch;
    p->paulis = paulis;
    p->n_slots = n_slots;
    p->tmats = static_cast<const typename std::remove_pointer<decltype(p->tmats)>::type*>(tmats);
    return true;
  };
  if (dtype == SC_C64) {
    SweepParams<float> p;
    if (!fill(&p)) return cudaErrorInvalidValue;
    return launch_t<float>(states, p, err, sm_count, s);
  }
  SweepParams<double> p;
  if (!fill(&p)) return cudaErrorInvalidValue;
  return launch_t<double>(states, p, err, sm_count, s);
}

bool adjoint_plan_supported(const Plan& plan) {
  if (!plan.ok || !plan.restore.empty()) return false;
  for (const SwSweep& sw : plan.sweeps) {
    if (sw.nr != 3 || sw.T - sw.nr < 5 || sw.T - sw.nr > 8 || sw.relayout) return false;
    if (!(sw.scale_re == 1.0 && sw.scale_im == 0.0)) return false;
    for (int g = sweep_first_gate(plan, sw); g < plan.stages[sw.s1 - 1].g1; ++g) {
      switch (plan.gates[g].kind) {
        case SK_G1: case SK_X: case SK_SWAP: case SK_D1: case SK_D2: case SK_DP:
        case SK_CX: case SK_DPR: case SK_G1ALL: case SK_D1R: case SK_X0: case SK_CX0: case SK_DTAB:
        case SK_PROBE: case SK_D1H:
          break;
        case SK_ROTL:  // NR = 3: masks of three register bits
          if (plan.gates[g].a & ~7) return false;
          break;
        default: return false;
      }
    }
  }
  return true;
}

namespace {

template <typename R>
cudaError_t launch_adjoint_t(void* psi, void* lam, const Plan& plan, size_t k, double* partial,
                             int max_ctas, double* grad, int sm_count, cudaStream_t s) {
  using A = typename Amp<R>::type;
  SweepParams<R> p;
  if (!fill_params(plan, k, &p, false) || p.nr != 3) return cudaErrorInvalidValue;
  // probe records carry the gradient slot; the kernel wants the local probe index
  ProbeSlots slots;
  int n_probes = 0;
  const int ng = p.stages[p.n_stages - 1].g1;
  for (int g = 0; g < ng; ++g) {
    if (p.gates[g].kind != SK_PROBE) continue;
    if (n_probes >= kSweepMaxGates) return cudaErrorInvalidValue;
    slots.slot[n_probes] = p.gates[g].b;
    p.gates[g].b = n_probes++;
  }
  const int threads = 1 << (p.T - p.nr);
  if (threads < 32 || threads > 256) return cudaErrorInvalidValue;
  // 256-thread tiles at two CTAs per SM (128 registers); smaller tiles at three
  // (170 registers: the two states' registers without spills)
  const size_t smem = 2 * (sizeof(A) << p.T) + sizeof(double) * (size_t)n_probes * (threads / 32);
  // the lite record switch when every record of the sweep is one of its kinds
  bool lite = true;
  for (int st = 0; st < p.n_stages; ++st)
    for (int g = p.stages[st].g0; g < p.stages[st].g1; ++g) lite = lite && adjoint_lite_kind(p.gates[g].kind);
  if (const char* v = getenv("STATECRAFT_B200_ADJOINT_LITE")) lite = lite && atoi(v) != 0;
  auto kern = threads == 256 ? (lite ? k_adjoint_sweep<R, 3, 256, 2, true> : k_adjoint_sweep<R, 3, 256, 2, false>)
                             : (lite ? k_adjoint_sweep<R, 3, 128, 3, true> : k_adjoint_sweep<R, 3, 128, 3, false>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  const int64_t grid =
      std::max<int64_t>(1, std::min<int64_t>({p.tiles, (int64_t)sm_count * std::max(per_sm, 1),
                                              (int64_t)max_ctas}));
  kern<<<(unsigned)grid, threads, smem, s>>>(static_cast<A*>(psi), static_cast<A*>(lam), p,
                                              partial, n_probes);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (n_probes > 0) {
    k_probe_reduce<<<1, 128, 0, s>>>(partial, (int)grid, n_probes, slots, grad);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace

cudaError_t launch_adjoint_sweep(int dtype, void* psi, void* lam, const Plan& plan, size_t k,
                                 double* partial, int max_ctas, double* grad, int sm_count,
                                 cudaStream_t s) {
  if (dtype == SC_C64)
    return launch_adjoint_t<float>(psi, lam, plan, k, partial, max_ctas, grad, sm_count, s);
  return launch_adjoint_t<double>(psi, lam, plan, k, partial, max_ctas, grad, sm_count, s);
}

}  // namespace sc
