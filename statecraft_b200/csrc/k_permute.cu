// In-place permutation of physical qubit bits.  Sweeps that moved qubits onto
// the low physical bits leave the state in a permuted layout; these passes bring
// it back to the identity layout the rest of the library (sampling, expectation
// values, state read-out) works in.
//
// A tile is the 2^nbits amplitudes that differ in the permuted bits (plus the low
// bits, so both the reads and the writes are contiguous runs); the bit set is
// closed under the permutation, so a tile reads and writes the same addresses and
// the pass is in place.  A persistent CTA loads a tile into shared memory, then
// writes every output element from the element it comes from.
#include <algorithm>
#include <mutex>

#include "sc_device.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

struct PermParams {
  int32_t nbits;
  int32_t pad;
  int64_t tiles;
  int8_t bits[SW_PERM_MAX_BITS];
  int8_t src[SW_PERM_MAX_BITS];
  // shared-memory swizzle: tile element i sits in slot i ^ (XOR of swz[k] over the
  // set bits k of i); swz[k] only touches the bits that select a bank group
  uint8_t swz[SW_PERM_MAX_BITS];
};

constexpr int kPermThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kPermThreads)
    k_permute(typename Amp<R>::type* __restrict__ st, const __grid_constant__ PermParams p) {
  using A = typename Amp<R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // spread / source tables split into the low and high 6 bits of the tile index
  uint32_t* const addr_lo = reinterpret_cast<uint32_t*>(smem_raw);
  uint32_t* const addr_hi = addr_lo + 64;
  uint32_t* const src_lo = addr_hi + 64;
  uint32_t* const src_hi = src_lo + 64;
  uint32_t* const swz_lo = src_hi + 64;
  uint32_t* const swz_hi = swz_lo + 64;
  A* const tile = reinterpret_cast<A*>(swz_hi + 64);
  const uint32_t tid = threadIdx.x;
  if (tid < 64) {
    uint32_t alo = 0, ahi = 0, slo = 0, shi = 0, zlo = 0, zhi = 0;
    for (int k = 0; k < p.nbits; ++k) {
      const uint32_t lo_bit = (k < 6) ? ((tid >> k) & 1u) : 0u;
      const uint32_t hi_bit = (k >= 6) ? ((tid >> (k - 6)) & 1u) : 0u;
      alo |= lo_bit << p.bits[k];
      ahi |= hi_bit << p.bits[k];
      slo |= lo_bit << p.src[k];
      shi |= hi_bit << p.src[k];
      zlo ^= lo_bit ? (uint32_t)p.swz[k] : 0u;
      zhi ^= hi_bit ? (uint32_t)p.swz[k] : 0u;
    }
    addr_lo[tid] = alo;
    addr_hi[tid] = ahi;
    src_lo[tid] = slo;
    src_hi[tid] = shi;
    swz_lo[tid] = zlo;
    swz_hi[tid] = zhi;
  }
  __syncthreads();
  auto slot = [&](uint32_t i) { return i ^ swz_lo[i & 63u] ^ swz_hi[i >> 6]; };
  const uint32_t tsize = 1u << p.nbits;
  for (int64_t t = blockIdx.x; t < p.tiles; t += gridDim.x) {
    uint64_t base = (uint64_t)t;
#pragma unroll 1
    for (int k = 0; k < p.nbits; ++k) base = insert_zero64(base, p.bits[k]);
    A* const g = st + base;
    for (uint32_t e = tid; e < tsize; e += kPermThreads)
      tile[slot(e)] = g[addr_lo[e & 63u] | addr_hi[e >> 6]];
    __syncthreads();
    for (uint32_t o = tid; o < tsize; o += kPermThreads)
      g[addr_lo[o & 63u] | addr_hi[o >> 6]] = tile[slot(src_lo[o & 63u] | src_hi[o >> 6])];
    __syncthreads();
  }
}

std::mutex g_perm_mu;
bool g_perm_attr[2] = {false, false};

template <typename R>
cudaError_t launch_t(void* state, int n, const SwPerm& perm, int sm_count, cudaStream_t s) {
  using A = typename Amp<R>::type;
  if (perm.nbits < 1 || perm.nbits > SW_PERM_MAX_BITS || perm.nbits > n)
    return cudaErrorInvalidValue;
  PermParams p;
  p.nbits = perm.nbits;
  p.pad = 0;
  p.tiles = 1LL << (n - perm.nbits);
  for (int k = 0; k < SW_PERM_MAX_BITS; ++k) {
    p.bits[k] = perm.bits[k];
    p.src[k] = perm.src[k];
    p.swz[k] = 0;
  }
  // A 128-byte shared-memory row holds W = 8 (complex128) or 16 (complex64)
  // elements; lanes that access together (W of them) differ in tile bits 0..w-1
  // on the load and in bits src[0..w-1] on the permuted read.  Give each of those
  // source bits at or above w a bank-group vector that completes a basis with
  // the others, so both phases are conflict-free.
  {
    const int w = sizeof(A) == 16 ? 3 : 4;
    uint32_t used = 0;  // span of the bank-group vectors assigned so far (as a set of unit bits)
    int pending[4];
    int np = 0;
    for (int k = 0; k < w && k < perm.nbits; ++k) {
      const int b = perm.src[k];
      if (b < w) used |= 1u << b;
      else pending[np++] = b;
    }
    for (int i = 0; i < np; ++i) {
      int u = 0;
      while (u < w && ((used >> u) & 1u)) ++u;
      if (u >= w) break;
      p.swz[pending[i]] = (uint8_t)(1u << u);
      used |= 1u << u;
    }
  }
  const size_t smem = 6 * 64 * sizeof(uint32_t) + (sizeof(A) << perm.nbits);
  auto kern = k_permute<R>;
  {
    std::lock_guard<std::mutex> lk(g_perm_mu);
    const int di = sizeof(R) == 4 ? 1 : 0;
    if (!g_perm_attr[di]) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(6 * 64 * sizeof(uint32_t) +
                                                 (sizeof(A) << SW_PERM_MAX_BITS)));
      if (e != cudaSuccess) return e;
      g_perm_attr[di] = true;
    }
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPermThreads, smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = std::min<int64_t>(p.tiles, (int64_t)sm_count * std::max(per_sm, 1));
  kern<<<(unsigned)grid, kPermThreads, smem, s>>>(static_cast<A*>(state), p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_permute(int dtype, void* state, int n, const SwPerm& perm, int sm_count,
                           cudaStream_t s) {
  if (dtype == SC_C64) return launch_t<float>(state, n, perm, sm_count, s);
  return launch_t<double>(state, n, perm, sm_count, s);
}

}  // namespace sc
