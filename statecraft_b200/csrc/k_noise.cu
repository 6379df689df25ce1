// Monte-Carlo Kraus trajectory step on the device.
//
// Reference (StatevectorEngine.java:463-600): for each Kraus operator K_i one full
// sweep computes ||K_i psi||^2; one draw rng.nextDouble(total) picks i; K_i is
// applied; a LASSQ norm sweep and a scale sweep renormalise when |norm - 1| > 1e-12.
// Here one read sweep computes every branch weight at once (FP64 partial sums per
// CTA), a one-thread kernel sums them in a fixed order, validates them, draws the
// uniform from the noise SplitMix64 stream and writes K_i / sqrt(w_i) (the norm
// after applying K_i is w_i) to device memory, and one read-write sweep applies
// it.  Two sweeps per channel application instead of seven, and no host round trip.
#include <algorithm>
#include <cfloat>

#include "sc_device.cuh"
#include "sc_internal.h"
#include "sc_noise.h"

namespace sc {

namespace {

constexpr int kThreads = 256;

template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_kraus_weights(const typename Amp<R>::type* __restrict__ st, int n, KrausArgs a,
                    double* __restrict__ partial) {
  __shared__ double red[kThreads / 32][SC_MAX_KRAUS];
  double w[SC_MAX_KRAUS];
#pragma unroll
  for (int k = 0; k < SC_MAX_KRAUS; ++k) w[k] = 0.0;
  const uint64_t pairs = 1ULL << (n - 1);
  const uint64_t stride = 1ULL << a.target;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero64(p, a.target);
    const auto v0 = st[i0], v1 = st[i0 + stride];
    const double a0r = v0.x, a0i = v0.y, a1r = v1.x, a1i = v1.y;
#pragma unroll
    for (int k = 0; k < SC_MAX_KRAUS; ++k) {
      if (k >= a.nk) break;
      const double* K = a.k[k];
      const double o0r = K[0] * a0r - K[1] * a0i + K[2] * a1r - K[3] * a1i;
      const double o0i = K[0] * a0i + K[1] * a0r + K[2] * a1i + K[3] * a1r;
      const double o1r = K[4] * a0r - K[5] * a0i + K[6] * a1r - K[7] * a1i;
      const double o1i = K[4] * a0i + K[5] * a0r + K[6] * a1i + K[7] * a1r;
      w[k] += (o0r * o0r + o0i * o0i) + (o1r * o1r + o1i * o1i);
    }
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < SC_MAX_KRAUS; ++k) {
    double v = w[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < SC_MAX_KRAUS) {
    double s = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) s += red[q][threadIdx.x];
    partial[blockIdx.x * SC_MAX_KRAUS + threadIdx.x] = s;
  }
}

__global__ void k_kraus_select(const double* __restrict__ partial, int nblocks, KrausArgs a,
                               uint64_t seed, uint64_t draw, NoiseDevState* ns) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ns->status != 0) return;
  double w[SC_MAX_KRAUS];
  double total = 0.0;
  for (int k = 0; k < a.nk; ++k) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b * SC_MAX_KRAUS + k];
    if (!isfinite(s) || s < 0.0) {
      ns->status = kNoiseBadWeight;
      ns->bad_draw = draw;
      return;
    }
    w[k] = s;
    total += s;
  }
  if (!isfinite(total) || total <= 1e-15) {
    ns->status = kNoiseBadTotal;
    ns->bad_draw = draw;
    return;
  }
  // SplittableRandom.nextDouble(bound)
  double u = splitmix_double(seed, draw) * total;
  if (u >= total) u = nextafter(total, -DBL_MAX);
  int idx = a.nk - 1;
  double cum = 0.0;
  for (int k = 0; k < a.nk; ++k) {
    cum += w[k];
    if (u < cum) {
      idx = k;
      break;
    }
  }
  const double nsq = w[idx];
  if (!isfinite(nsq) || nsq == 0.0) {
    ns->status = kNoiseBadNorm;
    ns->bad_draw = draw;
    return;
  }
  const double scale = (fabs(nsq - 1.0) > 1e-12) ? 1.0 / sqrt(nsq) : 1.0;
  for (int e = 0; e < 8; ++e) ns->matrix[e] = a.k[idx][e] * scale;
  ns->last_choice = idx;
  ns->choices[draw % kNoiseChoiceRing] = idx;
}

template <typename R>
__global__ void k_kraus_apply(typename Amp<R>::type* __restrict__ st, int n, int target,
                              const NoiseDevState* __restrict__ ns) {
  if (ns->status != 0) return;
  const R m00r = (R)ns->matrix[0], m00i = (R)ns->matrix[1], m01r = (R)ns->matrix[2],
          m01i = (R)ns->matrix[3];
  const R m10r = (R)ns->matrix[4], m10i = (R)ns->matrix[5], m11r = (R)ns->matrix[6],
          m11i = (R)ns->matrix[7];
  const uint64_t pairs = 1ULL << (n - 1);
  const uint64_t stride = 1ULL << target;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = insert_zero64(p, target);
    const auto a0 = st[i0], a1 = st[i0 + stride];
    st[i0] = cmac2(m00r, m00i, a0, m01r, m01i, a1);
    st[i0 + stride] = cmac2(m10r, m10i, a0, m11r, m11i, a1);
  }
}

// ---- batches of trajectories --------------------------------------------------
// States of 2^n amplitudes back to back; blockIdx.y is the state, blockIdx.x a slice
// of its amplitude pairs.  The chosen K / sqrt(w) of each state is not applied here:
// the batch's next sweep applies it (an SK_TMAT record).  A Kraus point whose
// predecessor's matrix is still pending on another qubit (the two records after a
// two-qubit gate) weighs the state with that matrix applied on the fly.

// the target qubit's reduced density matrix, accumulated over amplitude pairs
// (a0, a1): rho[0] += |a0|^2, rho[1] += |a1|^2, rho[2] + i rho[3] += a0 conj(a1)
__device__ __forceinline__ void rho_add(double a0r, double a0i, double a1r, double a1i,
                                        double* rho) {
  rho[0] += a0r * a0r + a0i * a0i;
  rho[1] += a1r * a1r + a1i * a1i;
  rho[2] += a0r * a1r + a0i * a1i;
  rho[3] += a0i * a1r - a0r * a1i;
}

constexpr int kRho = 4;

template <typename R>
__global__ void __launch_bounds__(kThreads)
    k_kraus_rho_batch(const typename Amp<R>::type* __restrict__ states, int n, int target,
                      int pend_q, const R* __restrict__ pend, const int32_t* __restrict__ status,
                      double* __restrict__ partial) {
  __shared__ double red[kThreads / 32][kRho];
  const uint64_t t = blockIdx.y;
  const typename Amp<R>::type* st = states + (t << n);
  double rho[kRho] = {0.0, 0.0, 0.0, 0.0};
  const uint64_t stride = 1ULL << target;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  if (status[t] == 0 && !pend) {
    // kUnroll pairs per thread and step, their loads issued together
    constexpr int kUnroll = 4;
    const uint64_t pairs = 1ULL << (n - 1);
    for (uint64_t p0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p0 < pairs;
         p0 += kUnroll * step) {
      typename Amp<R>::type v0[kUnroll], v1[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + u * step;
        if (p < pairs) {
          const uint64_t i0 = insert_zero64(p, target);
          v0[u] = st[i0];
          v1[u] = st[i0 + stride];
        }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (p0 + u * step >= pairs) break;
        rho_add(v0[u].x, v0[u].y, v1[u].x, v1[u].y, rho);
      }
    }
  } else if (status[t] == 0) {
    // the pending matrix M on qubit pend_q first: y[x][.] = sum_z M[x][z] v[z][.]
    const R* m = pend + t * 8;
    const double mr[4] = {(double)m[0], (double)m[2], (double)m[4], (double)m[6]};
    const double mi[4] = {(double)m[1], (double)m[3], (double)m[5], (double)m[7]};
    const uint64_t pstride = 1ULL << pend_q;
    const int lo = target < pend_q ? target : pend_q;
    const int hi = target < pend_q ? pend_q : target;
    constexpr int kUnroll = 2;
    const uint64_t quads = 1ULL << (n - 2);
    for (uint64_t q0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q0 < quads;
         q0 += kUnroll * step) {
      typename Amp<R>::type v[kUnroll][2][2];  // [pending bit][target bit]
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const uint64_t q = q0 + u * step;
        if (q < quads) {
          const uint64_t i0 = insert_zero64(insert_zero64(q, lo), hi);
          v[u][0][0] = st[i0];
          v[u][0][1] = st[i0 + stride];
          v[u][1][0] = st[i0 + pstride];
          v[u][1][1] = st[i0 + pstride + stride];
        }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (q0 + u * step >= quads) break;
#pragma unroll
        for (int x = 0; x < 2; ++x) {
          double yr[2], yi[2];
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const double z0r = v[u][0][b].x, z0i = v[u][0][b].y;
            const double z1r = v[u][1][b].x, z1i = v[u][1][b].y;
            yr[b] = mr[2 * x] * z0r - mi[2 * x] * z0i + mr[2 * x + 1] * z1r - mi[2 * x + 1] * z1i;
            yi[b] = mr[2 * x] * z0i + mi[2 * x] * z0r + mr[2 * x + 1] * z1i + mi[2 * x + 1] * z1r;
          }
          rho_add(yr[0], yi[0], yr[1], yi[1], rho);
        }
      }
    }
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kRho; ++k) {
    double v = rho[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kRho) {
    double sum = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) sum += red[q][threadIdx.x];
    partial[(t * gridDim.x + blockIdx.x) * kRho + threadIdx.x] = sum;
  }
}

// one thread per trajectory: the reduced density matrix summed in a fixed order,
// each branch weight ||K psi||^2 = sum over K's rows r of |K_r0|^2 rho00 + |K_r1|^2
// rho11 + 2 Re(K_r0 conj(K_r1) rho01), validated, the branch drawn from
// SplittableRandom(seeds[0] + t) (draw number `draw`) and K / sqrt(w) written to
// mats[t] (the amplitude type's reals); status[t] records the first failure of
// trajectory t
template <typename R>
__global__ void k_kraus_select_batch(const double* __restrict__ partial, int nblocks,
                                     KrausArgs a, const uint64_t* __restrict__ seeds,
                                     uint64_t draw, int64_t batch, R* __restrict__ mats,
                                     int32_t* __restrict__ choices, int64_t choice_stride,
                                     int32_t* __restrict__ status) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= batch || status[t] != 0) return;
  double rho[kRho] = {0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < nblocks; ++b)
    for (int q = 0; q < kRho; ++q) rho[q] += partial[((uint64_t)t * nblocks + b) * kRho + q];
  double w[SC_MAX_KRAUS];
  double total = 0.0;
  for (int k = 0; k < a.nk; ++k) {
    const double* K = a.k[k];
    double s = 0.0;
    for (int r = 0; r < 2; ++r) {
      const double xr = K[4 * r], xi = K[4 * r + 1], yr = K[4 * r + 2], yi = K[4 * r + 3];
      // K_r0 conj(K_r1)
      const double pr = xr * yr + xi * yi, pi = xi * yr - xr * yi;
      s += (xr * xr + xi * xi) * rho[0] + (yr * yr + yi * yi) * rho[1] +
           2.0 * (pr * rho[2] - pi * rho[3]);
    }
    if (!isfinite(s) || s < 0.0) {
      status[t] = kNoiseBadWeight;
      return;
    }
    w[k] = s;
    total += s;
  }
  if (!isfinite(total) || total <= 1e-15) {
    status[t] = kNoiseBadTotal;
    return;
  }
  double u = splitmix_double(seeds[0] + (uint64_t)t, draw) * total;
  if (u >= total) u = nextafter(total, -DBL_MAX);
  int idx = a.nk - 1;
  double cum = 0.0;
  for (int k = 0; k < a.nk; ++k) {
    cum += w[k];
    if (u < cum) {
      idx = k;
      break;
    }
  }
  const double nsq = w[idx];
  if (!isfinite(nsq) || nsq == 0.0) {
    status[t] = kNoiseBadNorm;
    return;
  }
  const double scale = (fabs(nsq - 1.0) > 1e-12) ? 1.0 / sqrt(nsq) : 1.0;
  for (int e = 0; e < 8; ++e) mats[t * 8 + e] = (R)(a.k[idx][e] * scale);
  choices[t * choice_stride] = idx;
}

}  // namespace

int noise_grid_batch(int n, int64_t batch, int sm_count) {
  const uint64_t pairs = 1ULL << (n - 1);
  const uint64_t most = (pairs + kThreads - 1) / kThreads;
  const uint64_t want = ((uint64_t)sm_count * 8 + (uint64_t)batch - 1) / (uint64_t)batch;
  return (int)std::max<uint64_t>(1, std::min(most, want));
}

cudaError_t launch_kraus_batch(int dtype, const void* states, int n, int64_t batch,
                               const KrausArgs& a, int pend_q, const void* pend,
                               const uint64_t* seeds, uint64_t draw, double* partial, void* mats,
                               int32_t* choices, int64_t choice_stride, int32_t* status,
                               int sm_count, cudaStream_t s) {
  if (batch < 1 || batch > 65535 || n < 2) return cudaErrorInvalidValue;
  if (pend && (pend_q < 0 || pend_q >= n || pend_q == a.target)) return cudaErrorInvalidValue;
  const int gx = noise_grid_batch(n, batch, sm_count);
  const dim3 grid((unsigned)gx, (unsigned)batch);
  const unsigned sel = (unsigned)((batch + 127) / 128);
  if (dtype == SC_C64) {
    k_kraus_rho_batch<float><<<grid, kThreads, 0, s>>>(
        static_cast<const float2*>(states), n, a.target, pend_q, static_cast<const float*>(pend),
        status, partial);
    k_kraus_select_batch<float><<<sel, 128, 0, s>>>(partial, gx, a, seeds, draw, batch,
                                                    static_cast<float*>(mats), choices,
                                                    choice_stride, status);
  } else {
    k_kraus_rho_batch<double><<<grid, kThreads, 0, s>>>(
        static_cast<const double2*>(states), n, a.target, pend_q,
        static_cast<const double*>(pend), status, partial);
    k_kraus_select_batch<double><<<sel, 128, 0, s>>>(partial, gx, a, seeds, draw, batch,
                                                     static_cast<double*>(mats), choices,
                                                     choice_stride, status);
  }
  return cudaGetLastError();
}

int noise_grid(int n, int sm_count) {
  const uint64_t pairs = 1ULL << (n - 1);
  const uint64_t blocks = (pairs + kThreads - 1) / kThreads;
  const uint64_t cap = (uint64_t)sm_count * 8;
  return (int)(blocks < cap ? blocks : cap);
}

cudaError_t launch_kraus_channel(int dtype, void* state, int n, const KrausArgs& a,
                                 uint64_t seed, uint64_t draw, double* partial,
                                 NoiseDevState* ns, int sm_count, cudaStream_t s) {
  const int grid = noise_grid(n, sm_count);
  if (dtype == SC_C64) {
    k_kraus_weights<float><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(state), n, a,
                                                     partial);
  } else {
    k_kraus_weights<double><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(state), n, a,
                                                      partial);
  }
  k_kraus_select<<<1, 32, 0, s>>>(partial, grid, a, seed, draw, ns);
  if (dtype == SC_C64)
    k_kraus_apply<float><<<grid, kThreads, 0, s>>>(static_cast<float2*>(state), n, a.target, ns);
  else
    k_kraus_apply<double><<<grid, kThreads, 0, s>>>(static_cast<double2*>(state), n, a.target,
                                                    ns);
  return cudaGetLastError();
}

}  // namespace sc
