// Fused tile-sweep kernel: one HBM read + one HBM write of every amplitude
// applies every gate the planner packed into the sweep.
//
// Tile: the 2^T amplitudes whose indices differ only in the tile qubits (the L
// lowest qubits, contiguous in memory, plus h high qubits).  A persistent CTA
// walks tiles.  Per tile it runs the sweep's stages; in stage s each thread holds
// 2^NR amplitudes in registers that differ in the stage's register positions
// R[0..NR-1], applies the stage's gates there, and the next stage re-distributes
// the tile through XOR-swizzled shared memory.  The first stage loads straight
// from HBM and the last stage stores straight to HBM: with R on high positions,
// the lanes of a warp walk the low (contiguous) positions, so every warp access is
// a contiguous 2^min(L,5)-amplitude run of 128-bit (c128) / 64-bit (c64) words.
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "sc_device.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

// local tile index -> global index bits (without the tile base)
__device__ __forceinline__ uint64_t spread(uint32_t x, const SwSweep& sw) {
  uint64_t g = x & ((1u << sw.L) - 1u);
  uint32_t hi = x >> sw.L;
  for (int k = 0; hi; ++k, hi >>= 1)
    if (hi & 1u) g |= 1ULL << sw.hq[k];
  return g;
}

__device__ __forceinline__ int bit_ref(int ref, uint32_t lidx, uint64_t base) {
  return ref >= 0 ? (int)((lidx >> ref) & 1u) : (int)((base >> (-ref - 1)) & 1ULL);
}

template <typename R, int NR, int A_>
__device__ __forceinline__ void g1(typename Amp<R>::type (&v)[1 << NR], const R* m,
                                   uint32_t l0, const uint32_t (&off)[1 << NR], uint32_t lmask) {
  const R m00r = m[0], m00i = m[1], m01r = m[2], m01i = m[3];
  const R m10r = m[4], m10i = m[5], m11r = m[6], m11i = m[7];
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & (1 << A_)) continue;
    constexpr int bit = 1 << A_;
    const int j1 = j | bit;
    if (lmask && (((l0 | off[j]) & lmask) != lmask)) continue;
    const auto a0 = v[j], a1 = v[j1];
    v[j] = cmac2(m00r, m00i, a0, m01r, m01i, a1);
    v[j1] = cmac2(m10r, m10i, a0, m11r, m11i, a1);
  }
}

template <typename R, int NR, int A_>
__device__ __forceinline__ void xswap(typename Amp<R>::type (&v)[1 << NR], uint32_t l0,
                                      const uint32_t (&off)[1 << NR], uint32_t lmask) {
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & (1 << A_)) continue;
    const int j1 = j | (1 << A_);
    if (lmask && (((l0 | off[j]) & lmask) != lmask)) continue;
    const auto t = v[j];
    v[j] = v[j1];
    v[j1] = t;
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

template <typename R, int NR, int A_, int B_>
__device__ __forceinline__ void rswap(typename Amp<R>::type (&v)[1 << NR]) {
#pragma unroll
  for (int j = 0; j < (1 << NR); ++j) {
    if (j & ((1 << A_) | (1 << B_))) continue;
    const int ja = j | (1 << A_), jb = j | (1 << B_);
    const auto t = v[ja];
    v[ja] = v[jb];
    v[jb] = t;
  }
}

template <int NR, typename F>
__device__ __forceinline__ void dispatch1(int a, F&& f) {
  switch (a) {
    case 0: f(std::integral_constant<int, 0>()); break;
    case 1: if constexpr (NR > 1) f(std::integral_constant<int, 1>()); break;
    case 2: if constexpr (NR > 2) f(std::integral_constant<int, 2>()); break;
    case 3: if constexpr (NR > 3) f(std::integral_constant<int, 3>()); break;
    default: break;
  }
}

template <int NR, typename F>
__device__ __forceinline__ void dispatch2(int a, int b, F&& f) {
  dispatch1<NR>(a, [&](auto ia) {
    dispatch1<NR>(b, [&](auto ib) {
      if constexpr (decltype(ia)::value != decltype(ib)::value) f(ia, ib);
    });
  });
}

// Block size is 2^(T - NR); the bound keeps >= 128 registers for NR >= 3.
template <typename R, int NR>
constexpr int sweep_max_threads() {
  return NR >= 4 ? (sizeof(R) == 8 ? 256 : 512) : (NR == 3 ? 512 : 1024);
}

template <typename R, int NR>
__global__ void __launch_bounds__(sweep_max_threads<R, NR>())
    k_sweep(typename Amp<R>::type* __restrict__ st, const SwSweep sw,
            const SwStage* __restrict__ stages, const SwGate* __restrict__ gates,
            const R* __restrict__ pool) {
  using A = typename Amp<R>::type;
  constexpr int NV = 1 << NR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* tile = reinterpret_cast<A*>(smem_raw);
  const uint32_t tid = threadIdx.x;

  for (int64_t t = blockIdx.x; t < sw.tiles; t += gridDim.x) {
    uint64_t base = (uint64_t)t << sw.L;
    for (int k = 0; k < sw.h; ++k) base = insert_zero64(base, sw.hq[k]);

    A v[NV];
    uint32_t l0 = 0;
    uint32_t off[NV];
    for (int s = sw.s0; s < sw.s1; ++s) {
      const SwStage stg = stages[s];
      uint32_t nl0 = tid;
#pragma unroll
      for (int k = 0; k < NR; ++k) nl0 = insert_zero32(nl0, stg.R[k]);
      uint32_t noff[NV];
#pragma unroll
      for (int j = 0; j < NV; ++j) {
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (j & (1 << k)) o |= 1u << stg.R[k];
        noff[j] = o;
      }
      if (s == sw.s0) {
        const uint64_t g0 = base | spread(nl0, sw);
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = st[g0 | spread(noff[j], sw)];
      } else {
        __syncthreads();  // previous readers of the tile are done
#pragma unroll
        for (int j = 0; j < NV; ++j) tile[swz<R>(l0 | off[j])] = v[j];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = tile[swz<R>(nl0 | noff[j])];
      }
      l0 = nl0;
#pragma unroll
      for (int j = 0; j < NV; ++j) off[j] = noff[j];

      for (int gi = stg.g0; gi < stg.g1; ++gi) {
        const SwGate g = gates[gi];
        if ((base & g.gmask) != g.gmask) continue;
        const R* m = pool + g.moff;
        switch (g.kind) {
          case SK_G1:
            dispatch1<NR>(g.a, [&](auto ia) { g1<R, NR, decltype(ia)::value>(v, m, l0, off, g.lmask); });
            break;
          case SK_X:
            dispatch1<NR>(g.a, [&](auto ia) { xswap<R, NR, decltype(ia)::value>(v, l0, off, g.lmask); });
            break;
          case SK_G2:
            if constexpr (NR > 1)
              dispatch2<NR>(g.a, g.b, [&](auto ia, auto ib) {
                g2<R, NR, decltype(ia)::value, decltype(ib)::value>(v, m);
              });
            break;
          case SK_SWAP:
            if constexpr (NR > 1)
              dispatch2<NR>(g.a, g.b, [&](auto ia, auto ib) {
                constexpr int kA = decltype(ia)::value;
                constexpr int kB = decltype(ib)::value;
                if constexpr (kA < kB)
                  rswap<R, NR, kA, kB>(v);
                else
                  rswap<R, NR, kB, kA>(v);
              });
            break;
          case SK_D1: {
            const R d0r = m[0], d0i = m[1], d1r = m[2], d1i = m[3];
#pragma unroll
            for (int j = 0; j < NV; ++j) {
              const uint32_t li = l0 | off[j];
              if ((li & g.lmask) != g.lmask) continue;
              const int bit = bit_ref(g.a, li, base);
              v[j] = bit ? cmul(d1r, d1i, v[j]) : cmul(d0r, d0i, v[j]);
            }
            break;
          }
          case SK_D2: {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
              const uint32_t li = l0 | off[j];
              const int k = (bit_ref(g.a, li, base) << 1) | bit_ref(g.b, li, base);
              v[j] = cmul(m[2 * k], m[2 * k + 1], v[j]);
            }
            break;
          }
          default: break;
        }
      }
    }
    const uint64_t g0 = base | spread(l0, sw);
#pragma unroll
    for (int j = 0; j < NV; ++j) st[g0 | spread(off[j], sw)] = v[j];
  }
}

struct LaunchCache {
  std::mutex mu;
  bool attr_set[2][SW_MAX_NR + 1] = {};
};
LaunchCache g_cache;

template <typename R, int NR>
cudaError_t launch_nr(void* state, const SwSweep& sw, const DevPlan& dp, int sm_count,
                      cudaStream_t s) {
  using A = typename Amp<R>::type;
  auto kern = k_sweep<R, NR>;
  const int di = std::is_same<R, float>::value ? 1 : 0;
  {
    std::lock_guard<std::mutex> lk(g_cache.mu);
    if (!g_cache.attr_set[di][NR]) {
      cudaError_t e =
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return e;
      g_cache.attr_set[di][NR] = true;
    }
  }
  const int threads = 1 << (sw.T - NR);
  if (threads > sweep_max_threads<R, NR>()) return cudaErrorInvalidConfiguration;
  const size_t smem = (sw.s1 - sw.s0 > 1) ? (sizeof(A) << sw.T) : 0;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  per_sm = std::max(per_sm, 1);
  const int64_t grid = std::min<int64_t>(sw.tiles, (int64_t)sm_count * per_sm);
  kern<<<(unsigned)grid, threads, smem, s>>>(static_cast<A*>(state), sw, dp.stages, dp.gates,
                                             static_cast<const R*>(dp.pool));
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_t(void* state, const SwSweep& sw, const DevPlan& dp, int sm_count,
                     cudaStream_t s) {
  switch (sw.nr) {
    case 1: return launch_nr<R, 1>(state, sw, dp, sm_count, s);
    case 2: return launch_nr<R, 2>(state, sw, dp, sm_count, s);
    case 3: return launch_nr<R, 3>(state, sw, dp, sm_count, s);
    case 4: return launch_nr<R, 4>(state, sw, dp, sm_count, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_sweep(int dtype, void* state, int n, const SwSweep& sw, const DevPlan& dp,
                         int sm_count, cudaStream_t s) {
  (void)n;
  return dtype == SC_C64 ? launch_t<float>(state, sw, dp, sm_count, s)
                         : launch_t<double>(state, sw, dp, sm_count, s);
}

}  // namespace sc
