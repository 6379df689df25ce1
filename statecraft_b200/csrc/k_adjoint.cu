// Kernels for adjoint differentiation (addition; no counterpart in the reference
// engine).  Method: Jones & Gacon, "Efficient calculation of gradients in classical
// simulations of variational quantum algorithms", arXiv:2009.02823 (2020).
//   lambda = H psi;  for gates k = N..1:  if G_k = exp(-i t/2 P):
//       dE/dt += Im <lambda | P | psi>;   psi <- G_k^dag psi;  lambda <- G_k^dag lambda
// Inner products and the Pauli-sum application accumulate in FP64.
#include <algorithm>

#include "sc_adjoint.h"
#include "sc_device.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void times_i_pow(int ny, double& r, double& i) {
  double tr;
  switch (ny & 3) {
    case 1: tr = -i; i = r; r = tr; break;
    case 2: r = -r; i = -i; break;
    case 3: tr = i; i = -r; r = tr; break;
    default: break;
  }
}

// out (+)= sum_k c_k P_k psi for up to kSumTerms terms in one pass: per amplitude the
// terms are summed in FP64 in order and `out` is written once (for 32 consecutive i
// the partners i ^ x_k stay within one aligned 32-block, so the reads coalesce)
constexpr int kSumTerms = 64;

struct PauliTerms {
  uint64_t x[kSumTerms], z[kSumTerms];
  double c[kSumTerms];
  int32_t count, accumulate;
};

template <typename R>
__global__ void k_pauli_sum(const typename Amp<R>::type* __restrict__ psi,
                            typename Amp<R>::type* __restrict__ out, int n,
                            const __grid_constant__ PauliTerms t) {
  const uint64_t dim = 1ULL << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    double sr = 0.0, si = 0.0;
    if (t.accumulate) {
      const auto o = out[i];
      sr = (double)o.x;
      si = (double)o.y;
    }
    for (int k = 0; k < t.count; ++k) {
      const uint64_t j = i ^ t.x[k];
      const auto a = psi[j];
      double r = a.x, im = a.y;
      if (__popcll(t.z[k] & j) & 1) {
        r = -r;
        im = -im;
      }
      times_i_pow(__popcll(t.x[k] & t.z[k]), r, im);
      sr = fma(t.c[k], r, sr);
      si = fma(t.c[k], im, si);
    }
    out[i] = make_amp<R>((R)sr, (R)si);
  }
}

// partial[block] = sum_i conj(lam_i) (P psi)_i  (complex)
template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_pauli_inner(const typename Amp<R>::type* __restrict__ lam,
                  const typename Amp<R>::type* __restrict__ psi, int n, uint64_t x, uint64_t z,
                  double2* __restrict__ partial) {
  __shared__ double red_r[kThreads / 32], red_i[kThreads / 32];
  const int ny = __popcll(x & z) & 3;
  const uint64_t dim = 1ULL << n;
  double ar = 0.0, ai = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = i ^ x;
    const auto p = psi[j];
    double pr = p.x, pi = p.y;
    if (__popcll(z & j) & 1) {
      pr = -pr;
      pi = -pi;
    }
    times_i_pow(ny, pr, pi);
    const auto l = lam[i];
    const double lr = l.x, li = l.y;
    ar += lr * pr + li * pi;
    ai += lr * pi - li * pr;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ar += __shfl_xor_sync(0xffffffffu, ar, o);
    ai += __shfl_xor_sync(0xffffffffu, ai, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red_r[threadIdx.x >> 5] = ar;
    red_i[threadIdx.x >> 5] = ai;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) {
      sr += red_r[k];
      si += red_i[k];
    }
    partial[blockIdx.x] = make_double2(sr, si);
  }
}

// grad[slot] += Im(sum of partials)   (one thread; fixed order)
__global__ void k_accumulate_grad(const double2* __restrict__ partial, int nblocks,
                                  double* __restrict__ grad, int slot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double si = 0.0;
  for (int b = 0; b < nblocks; ++b) si += partial[b].y;
  grad[slot] += si;
}

int blocks_for(int n, int sm_count) {
  const uint64_t dim = 1ULL << n;
  uint64_t b = (dim + kThreads - 1) / kThreads;
  const uint64_t cap = (uint64_t)sm_count * 8;
  return (int)(b > cap ? cap : b);
}

}  // namespace

int adjoint_partial_blocks(int n, int sm_count) { return blocks_for(n, sm_count); }

cudaError_t launch_pauli_sum(int dtype, const void* psi, void* out, int n, const uint64_t* x,
                             const uint64_t* z, const double* c, int64_t count, int sm_count,
                             cudaStream_t s) {
  const int grid = blocks_for(n, sm_count);
  for (int64_t k0 = 0; k0 < count; k0 += kSumTerms) {
    PauliTerms t;
    t.count = (int32_t)std::min<int64_t>(kSumTerms, count - k0);
    t.accumulate = k0 > 0;
    for (int k = 0; k < t.count; ++k) {
      t.x[k] = x[k0 + k];
      t.z[k] = z[k0 + k];
      t.c[k] = c[k0 + k];
    }
    if (dtype == SC_C64)
      k_pauli_sum<float><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(psi),
                                                   static_cast<float2*>(out), n, t);
    else
      k_pauli_sum<double><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(psi),
                                                    static_cast<double2*>(out), n, t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_inner(int dtype, const void* lam, const void* psi, int n, double2* partial,
                         int sm_count, cudaStream_t s) {
  const int grid = blocks_for(n, sm_count);
  if (dtype == SC_C64)
    k_pauli_inner<float><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(lam),
                                                   static_cast<const float2*>(psi), n, 0, 0,
                                                   partial);
  else
    k_pauli_inner<double><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(lam),
                                                    static_cast<const double2*>(psi), n, 0, 0,
                                                    partial);
  return cudaGetLastError();
}

cudaError_t launch_generator_grad(int dtype, const void* lam, const void* psi, int n, uint64_t x,
                                  uint64_t z, double2* partial, double* grad, int slot,
                                  int sm_count, cudaStream_t s) {
  const int grid = blocks_for(n, sm_count);
  if (dtype == SC_C64)
    k_pauli_inner<float><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(lam),
                                                   static_cast<const float2*>(psi), n, x, z,
                                                   partial);
  else
    k_pauli_inner<double><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(lam),
                                                    static_cast<const double2*>(psi), n, x, z,
                                                    partial);
  k_accumulate_grad<<<1, 32, 0, s>>>(partial, grid, grad, slot);
  return cudaGetLastError();
}

}  // namespace sc
