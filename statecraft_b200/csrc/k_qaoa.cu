// Batched QAOA ring-ansatz kernels: many instances of uneven size in one launch.
//
// Work items are (instance, tile) pairs laid end to end over the instance list;
// persistent CTAs walk them.  A tile is 2^12 amplitudes held in shared memory.
// In a tile, each thread keeps 2^NR amplitudes in registers that differ in one
// "group" of NR tile bits; the RX layer is applied group by group, moving the
// tile between register layouts through shared memory (XOR-swizzled slots, so
// every exchange is free of bank conflicts).  The cost phase of a layer is one
// lookup in a per-instance table of n + 1 phases.
//
//   whole mode (n <= 12): init, every layer and the energy in one item
//   low / high passes (n > 12): the circuit is split into p + 1 passes, each one
//     HBM read + write of the state (the first writes only, the last reads only):
//       P0 (low)  : H^n|0>, phase 0, RX 0 on qubits 0..11
//       Pk        : RX k-1 on its half, phase k, RX k on its half (halves alternate)
//       Pp        : RX p-1 on its half, energy
//     RX layers on the two halves commute, so this order is the circuit's.
//
// Energies: sum_x |a_x|^2 (n - 2 popcount(x ^ rotr(x))) in FP64 per item, summed
// per instance in item order by launch_qaoa_reduce (deterministic).
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "sc_device.cuh"
#include "sc_internal.h"
#include "sc_qaoa.h"

namespace sc {

namespace {

constexpr int kQT = kQaoaTileQubits;
constexpr uint32_t kTile = 1u << kQT;

template <typename R>
constexpr int qaoa_banks() {
  return sizeof(typename Amp<R>::type) == 16 ? 8 : 16;  // amplitudes per 128-byte row
}

// shared-memory slot of tile element e: the bank-group bits are XORed with the
// bits just above the register group width, which separates the lanes of every
// register layout the kernel uses
template <typename R, int NR>
__device__ __forceinline__ uint32_t qslot(uint32_t e) {
  return e ^ ((e >> NR) & (uint32_t)(qaoa_banks<R>() - 1));
}

__host__ __device__ constexpr size_t qaoa_smem_bytes(size_t amp_bytes, int p, bool db) {
  return (db ? 2 : 1) * amp_bytes * kTile + (size_t)p * (kQaoaMaxQubits + 1) * amp_bytes +
         2 * kQaoaMaxLayers * (amp_bytes / 2) + 64 * sizeof(double);
}

template <int V>
using IC = std::integral_constant<int, V>;

// f(IC<I>) for I = 0 .. N-1 (ascending) at compile time
template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F& f) {
  if constexpr (I < N) {
    f(IC<I>());
    static_for<I + 1, N>(f);
  }
}

// runs f(IC<g>) for the runtime group index g
template <int NG, typename F>
__device__ __forceinline__ void with_group(int g, F&& f) {
  if constexpr (NG > 0) if (g == 0) { f(IC<0>()); return; }
  if constexpr (NG > 1) if (g == 1) { f(IC<1>()); return; }
  if constexpr (NG > 2) if (g == 2) { f(IC<2>()); return; }
  if constexpr (NG > 3) if (g == 3) { f(IC<3>()); return; }
}

// MB: resident CTAs per SM the register allocation is sized for; DB: double-
// buffered tiles (the next item's amplitudes stream in while this item computes);
// MODE: kQaoaWhole / kQaoaLow / kQaoaHigh.
//
// Register group G holds tile bits [G*NR, G*NR+NR); thread t fills the other
// bits in order.  Both the shared-memory swizzle and the tile -> state index map
// are XOR-linear over disjoint bits, so each register's slot and offset is the
// thread's group base XOR a compile-time constant.
template <typename R, int NR, int MB, bool DB, int MODE>
__global__ void __launch_bounds__(1 << (kQT - NR), MB)
    k_qaoa(QaoaLaunch a, QaoaPass pass) {
  using A = typename Amp<R>::type;
  constexpr int NV = 1 << NR;
  constexpr int NG = kQT / NR;
  constexpr int kThreads = 1 << (kQT - NR);
  static_assert(kQT % NR == 0, "register groups must tile the 12 tile bits");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* const tiles = reinterpret_cast<A*>(smem_raw);
  A* const ph = tiles + (DB ? 2 : 1) * kTile;
  R* const rxc = reinterpret_cast<R*>(ph + a.p * (kQaoaMaxQubits + 1));  // (t, form) per layer
  double* const red = reinterpret_cast<double*>(rxc + 2 * kQaoaMaxLayers);
  const uint32_t t = threadIdx.x;
  A* const st = static_cast<A*>(a.state);
  const bool loads = MODE != kQaoaWhole && !pass.init;

  // the thread's tile-element base of each register group and its swizzled slot
  uint32_t ebase[NG], sbase[NG];
#pragma unroll
  for (int G = 0; G < NG; ++G) {
    const int lb = G * NR;
    ebase[G] = (t & ((1u << lb) - 1u)) | ((t >> lb) << (lb + NR));
    sbase[G] = qslot<R, NR>(ebase[G]);
  }

  // instance lookup, cached: consecutive items of a CTA usually share an instance
  int c_idx = -1;
  int64_t c_beg = 0, c_end = 0;
  QaoaInst c_in;
  auto locate = [&](int64_t w, QaoaInst& in, uint32_t& tileno) {
    if (c_idx < 0 || w < c_beg || w >= c_end) {
      int lo = 0, hi = a.n_inst - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.item_prefix[mid] <= w) lo = mid;
        else hi = mid - 1;
      }
      c_idx = lo;
      c_beg = a.item_prefix[lo];
      c_end = a.item_prefix[lo + 1];
      c_in = a.inst[lo];
    }
    in = c_in;
    tileno = (uint32_t)(w - c_beg);
  };
  // tile element -> index in the instance's state (linear over disjoint bits)
  auto tmap = [](int n, uint32_t e) -> uint32_t {
    if constexpr (MODE == kQaoaHigh) {
      const int c = 2 * kQT - n;  // contiguous low qubits kept in a high-mode tile
      return (e & ((1u << c) - 1u)) | ((e >> c) << kQT);
    } else {
      (void)n;
      return e;
    }
  };
  auto tile_off = [](int n, uint32_t tileno) -> uint32_t {
    if constexpr (MODE == kQaoaLow) return tileno << kQT;
    else if constexpr (MODE == kQaoaHigh) return tileno << (2 * kQT - n);
    else return 0u;
  };
  constexpr int kTop = NG - 1;
  auto prefetch = [&](int64_t w, A* buf) {
    QaoaInst in;
    uint32_t tileno;
    locate(w, in, tileno);
    const A* src = st + in.amp_off + (tile_off(in.n, tileno) | tmap(in.n, ebase[kTop]));
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      const uint32_t J = (uint32_t)j << (kTop * NR);
      cp_async<sizeof(A)>(buf + (sbase[kTop] ^ qslot<R, NR>(J)), src + tmap(in.n, J));
    }
  };

  int ph_loaded = -1;  // instance whose phase / RX tables are in shared memory
  int64_t w = blockIdx.x;
  if constexpr (DB) {
    if (loads && w < a.n_items) prefetch(w, tiles);
    cp_async_commit();
  }
  for (uint32_t it = 0; w < a.n_items; w += gridDim.x, ++it) {
    A* const cur = tiles + (DB ? (it & 1u) : 0u) * kTile;
    A* const nxt = tiles + (DB ? ((it & 1u) ^ 1u) : 0u) * kTile;
    QaoaInst in;
    uint32_t tileno;
    locate(w, in, tileno);
    const int n = in.n;
    const uint32_t nmask = (n >= 32) ? 0xffffffffu : ((1u << n) - 1u);
    uint32_t smask;  // tile bits the RX layers act on
    if constexpr (MODE == kQaoaLow) smask = kTile - 1u;
    else if constexpr (MODE == kQaoaHigh) smask = (kTile - 1u) & ~((1u << (2 * kQT - n)) - 1u);
    else smask = nmask;
    const uint32_t toff = tile_off(n, tileno);

    __syncthreads();  // the previous item is done with the tables and both tiles
    if (in.orig != ph_loaded) {
      const int l0 = (MODE == kQaoaWhole) ? 0 : pass.d;
      const int nl = (MODE == kQaoaWhole) ? a.p : (pass.d >= 0 ? 1 : 0);
      const int cnt = nl * (n + 1);
      for (int i = t; i < cnt; i += kThreads) {
        const double* src = a.phase + 2 * (in.ph_off + (int64_t)l0 * (n + 1) + i);
        ph[i] = make_amp<R>((R)src[0], (R)src[1]);
      }
      for (int i = t; i < 2 * a.p; i += kThreads) rxc[i] = (R)a.cs[2 * (int64_t)in.orig * a.p + i];
      ph_loaded = in.orig;
      __syncthreads();
    }

    A v[NV];
    int gcur = kTop;
    if (loads) {
      if constexpr (DB) {
        cp_async_wait<0>();  // this thread's copies of the current item have landed
#pragma unroll
        for (int j = 0; j < NV; ++j)
          v[j] = cur[sbase[kTop] ^ qslot<R, NR>((uint32_t)j << (kTop * NR))];
        const int64_t wn = w + gridDim.x;
        if (wn < a.n_items) prefetch(wn, nxt);
        cp_async_commit();
      } else {
        const A* src = st + in.amp_off + (toff | tmap(n, ebase[kTop]));
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = src[tmap(n, (uint32_t)j << (kTop * NR))];
        // the next item's amplitudes into L2 while this one computes (no registers,
        // nothing to wait for): its loads then hit L2 instead of HBM
        const int64_t wn = w + gridDim.x;
        if (wn < a.n_items) {
          QaoaInst inn;
          uint32_t tn;
          locate(wn, inn, tn);
          const A* nsrc = st + inn.amp_off + (tile_off(inn.n, tn) | tmap(inn.n, ebase[kTop]));
#pragma unroll
          for (int j = 0; j < NV; ++j) prefetch_l2(nsrc + tmap(inn.n, (uint32_t)j << (kTop * NR)));
        }
      }
    }
    auto has = [&](int G) { return ((smask >> (G * NR)) & (uint32_t)(NV - 1)) != 0u; };
    // move the tile from the current register layout to group G
    auto go = [&](auto gto) {
      constexpr int G = decltype(gto)::value;
      if (gcur == G) return;
      __syncthreads();
      with_group<NG>(gcur, [&](auto gfrom) {
        constexpr int F = decltype(gfrom)::value;
#pragma unroll
        for (int j = 0; j < NV; ++j) cur[sbase[F] ^ qslot<R, NR>((uint32_t)j << (F * NR))] = v[j];
      });
      __syncthreads();
#pragma unroll
      for (int j = 0; j < NV; ++j) v[j] = cur[sbase[G] ^ qslot<R, NR>((uint32_t)j << (G * NR))];
      gcur = G;
    };
    // RX(2 beta) = [[c, -i s], [-i s, c]] up to a scalar: c (I - i t X) with
    // t = s / c when |c| >= |s| (form 0), else s (u I - i X) with u = c / s
    // (form 1); |t|, |u| <= 1.  One FMA per output component; the scalars of a
    // whole layer half are folded into the phase tables / final energy on the host.
    auto rx = [&](int l) {
      const R tq = rxc[2 * l];
      const bool form1 = rxc[2 * l + 1] != (R)0;
      const uint32_t rm = (smask >> (gcur * NR)) & (uint32_t)(NV - 1);
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        if (!((rm >> k) & 1u)) continue;
        if (!form1) {
#pragma unroll
          for (int j = 0; j < NV; ++j) {
            if (j & (1 << k)) continue;
            const A a0 = v[j], a1 = v[j | (1 << k)];
            // (I - i t X): n0 = a0 - i t a1, n1 = a1 - i t a0
            v[j] = make_amp<R>(fma(tq, a1.y, a0.x), fma(-tq, a1.x, a0.y));
            v[j | (1 << k)] = make_amp<R>(fma(tq, a0.y, a1.x), fma(-tq, a0.x, a1.y));
          }
        } else {
#pragma unroll
          for (int j = 0; j < NV; ++j) {
            if (j & (1 << k)) continue;
            const A a0 = v[j], a1 = v[j | (1 << k)];
            // (u I - i X): n0 = u a0 - i a1, n1 = u a1 - i a0
            v[j] = make_amp<R>(fma(tq, a0.x, a1.y), fma(tq, a0.y, -a1.x));
            v[j | (1 << k)] = make_amp<R>(fma(tq, a1.x, a0.y), fma(tq, a1.y, -a0.x));
          }
        }
      }
    };
    // k(x) = popcount(x ^ rotr_n(x)) is linear in x: k(base ^ J) = popc(X(base) ^ X(J))
    auto xk = [&](uint32_t g) { return (g ^ ((g >> 1) | ((g & 1u) << (n - 1)))) & nmask; };
    auto phase = [&](int slot_layer) {
      const A* tab = ph + slot_layer * (n + 1);
      with_group<NG>(gcur, [&](auto gg) {
        constexpr int G = decltype(gg)::value;
        const uint32_t x0 = xk(toff | tmap(n, ebase[G]));
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          const A f = tab[__popc(x0 ^ xk(tmap(n, (uint32_t)j << (G * NR))))];
          v[j] = cmul(f.x, f.y, v[j]);
        }
      });
    };
    auto lowest_has = [&]() {
      int G = 0;
      while (G < NG - 1 && !has(G)) ++G;
      return G;
    };
    auto init_regs = [&]() {
      const R amp0 = (R)rsqrt(ldexp(1.0, n));  // H^n |0>: every amplitude 2^(-n/2)
      with_group<NG>(gcur, [&](auto gg) {
        constexpr int G = decltype(gg)::value;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          const uint32_t e = ebase[G] | ((uint32_t)j << (G * NR));
          const bool valid = (MODE != kQaoaWhole) || ((e & ~nmask) == 0u);
          v[j] = make_amp<R>(valid ? amp0 : (R)0, (R)0);
        }
      });
    };
    auto visit_down = [&](int l) {
      auto f = [&](auto ii) {
        constexpr int G = NG - 1 - decltype(ii)::value;
        if (G <= gcur && has(G)) {
          go(IC<G>());
          rx(l);
        }
      };
      static_for<0, NG>(f);
    };
    auto visit_up = [&](int l) {
      auto f = [&](auto ii) {
        constexpr int G = decltype(ii)::value;
        if (G >= gcur && has(G)) {
          go(IC<G>());
          rx(l);
        }
      };
      static_for<0, NG>(f);
    };

    bool reduce = false;
    if constexpr (MODE == kQaoaWhole) {
      gcur = lowest_has();
      init_regs();
      for (int l = 0; l < a.p; ++l) {
        phase(l);
        if (gcur == lowest_has()) visit_up(l);
        else visit_down(l);
      }
      reduce = true;
    } else {
      if (pass.init) {
        gcur = lowest_has();
        init_regs();
      }
      if (pass.rx_a >= 0) visit_down(pass.rx_a);
      if (pass.d >= 0) phase(0);
      if (pass.rx_b >= 0) visit_up(pass.rx_b);
      reduce = pass.reduce != 0;
      if (!reduce) {
        go(IC<kTop>());
        A* dst = st + in.amp_off + (toff | tmap(n, ebase[kTop]));
#pragma unroll
        for (int j = 0; j < NV; ++j) dst[tmap(n, (uint32_t)j << (kTop * NR))] = v[j];
      }
    }

    if (reduce) {
      double e_acc = 0.0, n_acc = 0.0;
      with_group<NG>(gcur, [&](auto gg) {
        constexpr int G = decltype(gg)::value;
        const uint32_t x0 = xk(toff | tmap(n, ebase[G]));
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          const uint32_t J = (uint32_t)j << (G * NR);
          if (MODE == kQaoaWhole && ((ebase[G] | J) & ~nmask)) continue;
          const double re = (double)v[j].x, im = (double)v[j].y;
          const double p2 = re * re + im * im;
          e_acc += p2 * (double)(n - 2 * __popc(x0 ^ xk(tmap(n, J))));
          n_acc += p2;
        }
      });
      const double es = a.escale[in.orig];  // squared scalar of the last RX half
      e_acc *= es;
      n_acc *= es;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        e_acc += __shfl_xor_sync(0xffffffffu, e_acc, o);
        n_acc += __shfl_xor_sync(0xffffffffu, n_acc, o);
      }
      const int warp = t >> 5, lane = t & 31;
      __syncthreads();  // red[] of the previous item has been read
      if (lane == 0) {
        red[2 * warp] = e_acc;
        red[2 * warp + 1] = n_acc;
      }
      __syncthreads();
      if (t == 0) {
        double es = 0.0, ns = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
          es += red[2 * k];
          ns += red[2 * k + 1];
        }
        a.partials[2 * (a.part_base + w)] = es;
        a.partials[2 * (a.part_base + w) + 1] = ns;
      }
    }
  }
  if constexpr (DB) cp_async_wait<0>();
}

// one warp per instance sums its partial slots in order
__global__ void k_qaoa_reduce(const double* __restrict__ partials, const QaoaSpan* __restrict__ spans,
                              int64_t n_inst, double* __restrict__ energies,
                              double* __restrict__ norms) {
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n_inst) return;
  const QaoaSpan sp = spans[i];
  double e = 0.0, nn = 0.0;
  for (int64_t k = sp.begin + lane; k < sp.end; k += 32) {
    e += partials[2 * k];
    nn += partials[2 * k + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    nn += __shfl_xor_sync(0xffffffffu, nn, o);
  }
  if (lane == 0) {
    energies[i] = e;
    norms[i] = nn;
  }
}

std::mutex g_qaoa_mu;
bool g_qaoa_attr[2][kQaoaShapes][3] = {};

template <typename R, int NR, int MB, bool DB, int MODE>
cudaError_t set_attr(int shape) {
  std::lock_guard<std::mutex> lk(g_qaoa_mu);
  const int di = sizeof(R) == 4 ? 1 : 0;
  if (g_qaoa_attr[di][shape][MODE]) return cudaSuccess;
  const size_t most = qaoa_smem_bytes(sizeof(typename Amp<R>::type), kQaoaMaxLayers, DB);
  cudaError_t e = cudaFuncSetAttribute(k_qaoa<R, NR, MB, DB, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most);
  if (e == cudaSuccess) g_qaoa_attr[di][shape][MODE] = true;
  return e;
}

template <typename R, int NR, int MB, bool DB>
int max_ctas(int shape, int p) {
  if (set_attr<R, NR, MB, DB, kQaoaWhole>(shape) != cudaSuccess ||
      set_attr<R, NR, MB, DB, kQaoaLow>(shape) != cudaSuccess ||
      set_attr<R, NR, MB, DB, kQaoaHigh>(shape) != cudaSuccess)
    return 0;
  int per_sm = 0;
  const size_t smem = qaoa_smem_bytes(sizeof(typename Amp<R>::type), p, DB);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_qaoa<R, NR, MB, DB, kQaoaLow>,
                                                    1 << (kQT - NR), smem) != cudaSuccess)
    return 0;
  return per_sm;
}

template <typename R, int NR, int MB, bool DB, int MODE>
cudaError_t launch_mode(int shape, const QaoaLaunch& a, const QaoaPass& pass, int ctas_per_sm,
                        int sm_count, cudaStream_t s) {
  cudaError_t e = set_attr<R, NR, MB, DB, MODE>(shape);
  if (e != cudaSuccess) return e;
  const size_t smem = qaoa_smem_bytes(sizeof(typename Amp<R>::type), a.p, DB);
  const int64_t grid = std::min<int64_t>(a.n_items, (int64_t)sm_count * std::max(ctas_per_sm, 1));
  k_qaoa<R, NR, MB, DB, MODE><<<(unsigned)grid, 1 << (kQT - NR), smem, s>>>(a, pass);
  return cudaGetLastError();
}

template <typename R, int NR, int MB, bool DB>
cudaError_t launch_t(int shape, const QaoaLaunch& a, const QaoaPass& pass, int ctas_per_sm,
                     int sm_count, cudaStream_t s) {
  if (a.n_items <= 0) return cudaSuccess;
  switch (pass.mode) {
    case kQaoaWhole: return launch_mode<R, NR, MB, DB, kQaoaWhole>(shape, a, pass, ctas_per_sm, sm_count, s);
    case kQaoaLow: return launch_mode<R, NR, MB, DB, kQaoaLow>(shape, a, pass, ctas_per_sm, sm_count, s);
    case kQaoaHigh: return launch_mode<R, NR, MB, DB, kQaoaHigh>(shape, a, pass, ctas_per_sm, sm_count, s);
    default: return cudaErrorInvalidValue;
  }
}

// shape -> (register qubits NR, CTAs per SM the registers are sized for, double buffer)
template <typename F>
auto with_shape(int shape, F&& f) {
  switch (shape) {
    case 0: return f(IC<4>(), IC<2>(), std::false_type());
    case 1: return f(IC<4>(), IC<2>(), std::true_type());
    case 2: return f(IC<3>(), IC<1>(), std::false_type());
    default: return f(IC<3>(), IC<2>(), std::true_type());
  }
}

}  // namespace

int qaoa_shape_nr(int shape) { return shape <= 1 ? 4 : 3; }

cudaError_t launch_qaoa(int dtype, int shape, const QaoaLaunch& a, const QaoaPass& pass,
                        int ctas_per_sm, int sm_count, cudaStream_t s) {
  if (a.p < 1 || a.p > kQaoaMaxLayers || shape < 0 || shape >= kQaoaShapes)
    return cudaErrorInvalidValue;
  return with_shape(shape, [&](auto nr, auto mb, auto db) {
    constexpr int NR = decltype(nr)::value, MB = decltype(mb)::value;
    constexpr bool DB = decltype(db)::value;
    if (dtype == SC_C64) return launch_t<float, NR, MB, DB>(shape, a, pass, ctas_per_sm, sm_count, s);
    return launch_t<double, NR, MB, DB>(shape, a, pass, ctas_per_sm, sm_count, s);
  });
}

int qaoa_max_ctas_per_sm(int dtype, int shape, int p) {
  if (shape < 0 || shape >= kQaoaShapes) return 0;
  return with_shape(shape, [&](auto nr, auto mb, auto db) {
    constexpr int NR = decltype(nr)::value, MB = decltype(mb)::value;
    constexpr bool DB = decltype(db)::value;
    if (dtype == SC_C64) return max_ctas<float, NR, MB, DB>(shape, p);
    return max_ctas<double, NR, MB, DB>(shape, p);
  });
}

cudaError_t launch_qaoa_reduce(const double* partials, const QaoaSpan* spans, int64_t n_inst,
                               double* energies, double* norms, cudaStream_t s) {
  if (n_inst <= 0) return cudaSuccess;
  const int warps = 8;
  const int64_t blocks = (n_inst + warps - 1) / warps;
  k_qaoa_reduce<<<(unsigned)blocks, 32 * warps, 0, s>>>(partials, spans, n_inst, energies, norms);
  return cudaGetLastError();
}

}  // namespace sc
