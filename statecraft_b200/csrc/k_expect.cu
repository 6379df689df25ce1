// Pauli-string expectation values <psi|P|psi> in FP64 (addition: the reference
// engine has no expectation API).  P = i^{|x&z|} X^x Z^z acts as
// (P psi)_i = i^{ny} (-1)^{popcount(z & (i ^ x))} psi_{i ^ x}; a warp's
// i..i+31 map to the aligned block (i..i+31) ^ x, so both reads stay coalesced.
#include "sc_device.cuh"
#include "sc_internal.h"
#include "sc_noise.h"

namespace sc {

namespace {

constexpr int kThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_pauli_term(const typename Amp<R>::type* __restrict__ st, int n, uint64_t x, uint64_t z,
                 double* __restrict__ partial) {
  __shared__ double red[kThreads / 32];
  const int ny = __popcll(x & z) & 3;
  const uint64_t dim = 1ULL << n;
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = i ^ x;
    const auto ai = st[i];
    const auto aj = st[j];
    double pr = aj.x, pi = aj.y;
    if (__popcll(z & j) & 1) {
      pr = -pr;
      pi = -pi;
    }
    double qr, qi;
    switch (ny) {
      case 0: qr = pr; qi = pi; break;
      case 1: qr = -pi; qi = pr; break;
      case 2: qr = -pr; qi = -pi; break;
      default: qr = pi; qi = -pr; break;
    }
    acc += (double)ai.x * qr + (double)ai.y * qi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) s += red[k];
    partial[blockIdx.x] = s;
  }
}

__global__ void k_sum_rows(const double* __restrict__ partial, int rows, int cols,
                           double* __restrict__ out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double s = 0.0;
  for (int c = 0; c < cols; ++c) s += partial[(size_t)r * cols + c];
  out[r] = s;
}

}  // namespace

cudaError_t launch_pauli_terms(int dtype, const void* state, int n, int n_terms,
                               const uint64_t* xmask, const uint64_t* zmask, double* partial,
                               size_t partial_elems, double* out_terms, int sm_count,
                               cudaStream_t s) {
  const uint64_t dim = 1ULL << n;
  uint64_t blocks = (dim + kThreads - 1) / kThreads;
  const uint64_t cap = (uint64_t)sm_count * 8;
  if (blocks > cap) blocks = cap;
  if ((size_t)blocks * (size_t)n_terms > partial_elems) return cudaErrorMemoryAllocation;
  for (int t = 0; t < n_terms; ++t) {
    double* part = partial + (size_t)t * blocks;
    if (dtype == SC_C64)
      k_pauli_term<float><<<(unsigned)blocks, kThreads, 0, s>>>(
          static_cast<const float2*>(state), n, xmask[t], zmask[t], part);
    else
      k_pauli_term<double><<<(unsigned)blocks, kThreads, 0, s>>>(
          static_cast<const double2*>(state), n, xmask[t], zmask[t], part);
  }
  k_sum_rows<<<(n_terms + 127) / 128, 128, 0, s>>>(partial, n_terms, (int)blocks, out_terms);
  return cudaGetLastError();
}

int pauli_partial_cols(int n, int sm_count) {
  const uint64_t dim = 1ULL << n;
  uint64_t blocks = (dim + kThreads - 1) / kThreads;
  const uint64_t cap = (uint64_t)sm_count * 8;
  return (int)(blocks > cap ? cap : blocks);
}

}  // namespace sc
