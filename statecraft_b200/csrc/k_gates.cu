// One-kernel-per-gate path (fusion off) plus state initialisation and dtype
// conversion.  Each gate kernel is a grid-stride loop over the pairs / groups the
// reference loops over (StatevectorOps.java scalar paths) with 64-bit indices and
// 128-bit (double2) or 64-bit (float2) amplitude accesses.
#include <algorithm>

#include "sc_device.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

struct GateArgs {
  double m[32];
  uint64_t cmask;
  int32_t q0, q1;
};

constexpr int kThreads = 256;

int grid_for(int64_t work) {
  int64_t blocks = (work + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, 148LL * 32));
}

template <typename R>
__global__ void k_dense1(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  using A = typename Amp<R>::type;
  const R m00r = (R)g.m[0], m00i = (R)g.m[1], m01r = (R)g.m[2], m01i = (R)g.m[3];
  const R m10r = (R)g.m[4], m10i = (R)g.m[5], m11r = (R)g.m[6], m11i = (R)g.m[7];
  const uint64_t stride = 1ULL << g.q0;
  const uint64_t pairs = 1ULL << (n - 1);
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero64(p, g.q0);
    if ((i0 & g.cmask) != g.cmask) continue;
    const uint64_t i1 = i0 + stride;
    const A a0 = st[i0], a1 = st[i1];
    st[i0] = cmac2(m00r, m00i, a0, m01r, m01i, a1);
    st[i1] = cmac2(m10r, m10i, a0, m11r, m11i, a1);
  }
}

template <typename R>
__global__ void k_dense2(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  using A = typename Amp<R>::type;
  const int low = min(g.q0, g.q1), high = max(g.q0, g.q1);
  const uint64_t of = 1ULL << g.q0, os = 1ULL << g.q1;
  const uint64_t groups = 1ULL << (n - 2);
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < groups;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = insert_zero64(insert_zero64(q, low), high);
    const uint64_t idx[4] = {b, b | os, b | of, b | of | os};
    A a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = st[idx[k]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      A o;
      o.x = 0;
      o.y = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const R mr = (R)g.m[2 * (4 * r + c)], mi = (R)g.m[2 * (4 * r + c) + 1];
        o.x += mr * a[c].x - mi * a[c].y;
        o.y += mr * a[c].y + mi * a[c].x;
      }
      st[idx[r]] = o;
    }
  }
}

template <typename R>
__global__ void k_pairswap(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  using A = typename Amp<R>::type;
  const uint64_t stride = 1ULL << g.q0;
  const uint64_t pairs = 1ULL << (n - 1);
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero64(p, g.q0);
    if ((i0 & g.cmask) != g.cmask) continue;
    const A a0 = st[i0];
    st[i0] = st[i0 + stride];
    st[i0 + stride] = a0;
  }
}

template <typename R>
__global__ void k_swap(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  using A = typename Amp<R>::type;
  const int low = min(g.q0, g.q1), high = max(g.q0, g.q1);
  const uint64_t of = 1ULL << g.q0, os = 1ULL << g.q1;
  const uint64_t groups = 1ULL << (n - 2);
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < groups;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = insert_zero64(insert_zero64(q, low), high);
    const A f = st[b | of];
    st[b | of] = st[b | os];
    st[b | os] = f;
  }
}

// diag(d0, d1) on q0 where the controls are set; one thread per pair.
template <typename R>
__global__ void k_diag1(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  const R d0r = (R)g.m[0], d0i = (R)g.m[1], d1r = (R)g.m[2], d1i = (R)g.m[3];
  const uint64_t stride = 1ULL << g.q0;
  const uint64_t pairs = 1ULL << (n - 1);
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero64(p, g.q0);
    if ((i0 & g.cmask) != g.cmask) continue;
    st[i0] = cmul(d0r, d0i, st[i0]);
    st[i0 + stride] = cmul(d1r, d1i, st[i0 + stride]);
  }
}

template <typename R>
__global__ void k_diag2(typename Amp<R>::type* __restrict__ st, int n, GateArgs g) {
  const uint64_t dim = 1ULL << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int k = (int)(((i >> g.q0) & 1ULL) << 1 | ((i >> g.q1) & 1ULL));
    st[i] = cmul((R)g.m[2 * k], (R)g.m[2 * k + 1], st[i]);
  }
}

template <typename R>
__global__ void k_init_basis(typename Amp<R>::type* __restrict__ st, uint64_t dim,
                             uint64_t basis) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x)
    st[i] = make_amp<R>((R)(i == basis ? 1 : 0), (R)0);
}

__global__ void k_convert_in_c64(float2* __restrict__ st, const double2* __restrict__ src,
                                 uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = src[i];
    st[i] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void k_convert_out_c64(const float2* __restrict__ st, double2* __restrict__ dst,
                                  uint64_t count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float2 v = st[i];
    dst[i] = make_double2((double)v.x, (double)v.y);
  }
}

template <typename R>
cudaError_t launch_gate_t(void* state, int n, const PGate& pg, cudaStream_t s) {
  using A = typename Amp<R>::type;
  A* st = static_cast<A*>(state);
  GateArgs g;
  std::copy(pg.m, pg.m + 32, g.m);
  g.cmask = pg.cmask;
  g.q0 = pg.q0;
  g.q1 = pg.q1;
  const int64_t pairs = 1LL << (n - 1);
  switch (pg.kind) {
    case PK_DENSE1: k_dense1<R><<<grid_for(pairs), kThreads, 0, s>>>(st, n, g); break;
    case PK_DENSE2: k_dense2<R><<<grid_for(pairs / 2), kThreads, 0, s>>>(st, n, g); break;
    case PK_X: k_pairswap<R><<<grid_for(pairs), kThreads, 0, s>>>(st, n, g); break;
    case PK_SWAP: k_swap<R><<<grid_for(pairs / 2), kThreads, 0, s>>>(st, n, g); break;
    case PK_DIAG1: k_diag1<R><<<grid_for(pairs), kThreads, 0, s>>>(st, n, g); break;
    case PK_DIAG2: k_diag2<R><<<grid_for(2 * pairs), kThreads, 0, s>>>(st, n, g); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_gate(int dtype, void* state, int n, const PGate& g, cudaStream_t s) {
  return dtype == SC_C64 ? launch_gate_t<float>(state, n, g, s)
                         : launch_gate_t<double>(state, n, g, s);
}

cudaError_t launch_init_basis(int dtype, void* state, int n, uint64_t basis, cudaStream_t s) {
  const uint64_t dim = 1ULL << n;
  const int grid = grid_for((int64_t)dim);
  if (dtype == SC_C64)
    k_init_basis<float><<<grid, kThreads, 0, s>>>(static_cast<float2*>(state), dim, basis);
  else
    k_init_basis<double><<<grid, kThreads, 0, s>>>(static_cast<double2*>(state), dim, basis);
  return cudaGetLastError();
}

// |0..0> in each of `batch` n-qubit states stored back to back
template <typename R>
__global__ void k_init_batch(typename Amp<R>::type* st, uint64_t total, uint64_t dim_mask) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x)
    st[i] = make_amp<R>((i & dim_mask) == 0 ? (R)1 : (R)0, (R)0);
}

cudaError_t launch_init_batch(int dtype, void* states, int n, int64_t batch, cudaStream_t s) {
  const uint64_t total = (uint64_t)batch << n;
  const int grid = grid_for((int64_t)total);
  const uint64_t mask = (1ULL << n) - 1ULL;
  if (dtype == SC_C64)
    k_init_batch<float><<<grid, kThreads, 0, s>>>(static_cast<float2*>(states), total, mask);
  else
    k_init_batch<double><<<grid, kThreads, 0, s>>>(static_cast<double2*>(states), total, mask);
  return cudaGetLastError();
}

cudaError_t launch_convert_in(int dtype, void* state, const double* src, int64_t count,
                              cudaStream_t s) {
  if (dtype != SC_C64)
    return cudaMemcpyAsync(state, src, (size_t)count * 16, cudaMemcpyDeviceToDevice, s);
  k_convert_in_c64<<<grid_for(count), kThreads, 0, s>>>(
      static_cast<float2*>(state), reinterpret_cast<const double2*>(src), (uint64_t)count);
  return cudaGetLastError();
}

cudaError_t launch_convert_out(int dtype, const void* state, double* dst, int64_t count,
                               cudaStream_t s) {
  if (dtype != SC_C64)
    return cudaMemcpyAsync(dst, state, (size_t)count * 16, cudaMemcpyDeviceToDevice, s);
  k_convert_out_c64<<<grid_for(count), kThreads, 0, s>>>(
      static_cast<const float2*>(state), reinterpret_cast<double2*>(dst), (uint64_t)count);
  return cudaGetLastError();
}

}  // namespace sc
