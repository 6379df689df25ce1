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
  A* const tile = reinterpret_cast<A*>(src_hi + 64);
  const uint32_t tid = threadIdx.x;
  if (tid < 64) {
    uint32_t alo = 0, ahi = 0, slo = 0, shi = 0;
    for (int k = 0; k < p.nbits; ++k) {
      const uint32_t lo_bit = (k < 6) ? ((tid >> k) & 1u) : 0u;
      const uint32_t hi_bit = (k >= 6) ? ((tid >> (k - 6)) & 1u) : 0u;
      alo |= lo_bit << p.bits[k];
      ahi |= hi_bit << p.bits[k];
      slo |= lo_bit << p.src[k];
      shi |= hi_bit << p.src[k];
    }
    addr_lo[tid] = alo;
    addr_hi[tid] = ahi;
    src_lo[tid] = slo;
    src_hi[tid] = shi;
  }
  __syncthreads();
  const uint32_t tsize = 1u << p.nbits;
  for (int64_t t = blockIdx.x; t < p.tiles; t += gridDim.x) {
    uint64_t base = (uint64_t)t;
#pragma unroll 1
    for (int k = 0; k < p.nbits; ++k) base = insert_zero64(base, p.bits[k]);
    A* const g = st + base;
    for (uint32_t e = tid; e < tsize; e += kPermThreads)
      tile[e] = g[addr_lo[e & 63u] | addr_hi[e >> 6]];
    __syncthreads();
    for (uint32_t o = tid; o < tsize; o += kPermThreads)
      g[addr_lo[o & 63u] | addr_hi[o >> 6]] = tile[src_lo[o & 63u] | src_hi[o >> 6]];
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
  }
  const size_t smem = 4 * 64 * sizeof(uint32_t) + (sizeof(A) << perm.nbits);
  auto kern = k_permute<R>;
  {
    std::lock_guard<std::mutex> lk(g_perm_mu);
    const int di = sizeof(R) == 4 ? 1 : 0;
    if (!g_perm_attr[di]) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(4 * 64 * sizeof(uint32_t) +
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
