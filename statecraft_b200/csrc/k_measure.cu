// Measurement: marginal probabilities, FP64 prefix sums and per-shot search.
//
// Reference semantics (StatevectorEngine.java:229-338): probabilities over the
// measured qubits, rescaled by 1/sum when |sum - 1| > 1e-12, running sum with the
// last entry forced to 1.0, and per shot the first index whose cumulative value
// is >= u (u >= 1 -> last index).  Here the cumulative array is never
// materialised: pass A reduces chunks of CHUNK probabilities (FP64), pass B scans
// the chunk sums in one CTA, pass C gives each shot a warp that binary-searches
// the chunk prefixes and scans its chunk in FP64.  Uniforms are the reference's
// SplittableRandom(seed).nextDouble() sequence, computed per shot from (seed, k).
#include <cfloat>

#include "sc_device.cuh"
#include "sc_internal.h"
#include "sc_measure.h"

namespace sc {

namespace {

constexpr int kChunk = kSampleChunk;
constexpr int kThreadsA = 256;

template <typename R>
struct DirectSrc {
  const typename Amp<R>::type* st;
  __device__ __forceinline__ double operator()(uint64_t i) const {
    const auto a = st[i];
    const double re = (double)a.x, im = (double)a.y;
    return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
  }
};

struct ArraySrc {
  const double* p;
  __device__ __forceinline__ double operator()(uint64_t i) const { return p[i]; }
};

template <int THREADS>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int k = 0; k < THREADS / 32; ++k) s += red[k];
  }
  return s;  // valid in thread 0
}

// pass A: S[c] = sum of chunk c.  A batch of states of len_per entries each,
// stored back to back, has chunks_per chunks per state (chunk c of the whole
// array is chunk c % chunks_per of state c / chunks_per).
template <typename Src>
__global__ void __launch_bounds__(kThreadsA) k_chunk_sums(Src src, uint64_t len_per,
                                                          uint64_t chunks_per, double* sums,
                                                          uint64_t chunks) {
  __shared__ double red[kThreadsA / 32];
  for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
    const uint64_t st = c / chunks_per;
    const uint64_t b = (c - st * chunks_per) * kChunk;
    const uint64_t off = st * len_per;
    double acc = 0.0;
    for (int k = threadIdx.x; k < kChunk; k += kThreadsA) {
      const uint64_t i = b + k;
      if (i < len_per) acc += src(off + i);
    }
    const double s = block_sum<kThreadsA>(acc, red);
    if (threadIdx.x == 0) sums[c] = s;
  }
}

// pass B (one CTA of 1024 threads per state): total, scale, exclusive chunk prefixes
__global__ void __launch_bounds__(1024) k_chunk_scan(const double* sums, uint64_t chunks,
                                                     double* prefix, SampleScalars* out) {
  sums += blockIdx.x * chunks;
  prefix += blockIdx.x * chunks;
  out += blockIdx.x;
  __shared__ double part[1024];
  __shared__ double red[32];
  const uint64_t per = (chunks + 1023) / 1024;
  const uint64_t b = threadIdx.x * per;
  const uint64_t e = min(chunks, b + per);
  double local = 0.0;
  for (uint64_t c = b; c < e; ++c) local += sums[c];
  part[threadIdx.x] = local;
  const double total = block_sum<1024>(local, red);
  __shared__ double s_total, s_scale;
  if (threadIdx.x == 0) {
    s_total = total;
    s_scale = (fabs(total - 1.0) > 1e-12 && total != 0.0) ? 1.0 / total : 1.0;
    // exclusive scan of the per-thread partials (1024 adds, sequential, deterministic)
    double run = 0.0;
    for (int k = 0; k < 1024; ++k) {
      const double v = part[k];
      part[k] = run;
      run += v;
    }
    out->total = total;
    out->scale = s_scale;
    out->status = (total == 0.0 || !isfinite(total)) ? 1 : 0;
  }
  __syncthreads();
  const double scale = s_scale;
  double run = part[threadIdx.x];
  for (uint64_t c = b; c < e; ++c) {
    prefix[c] = run * scale;
    run += sums[c];
  }
}

// pass C: one warp per shot.  In a batch, shot g belongs to state g / shots_per and
// draws the (g % shots_per)-th uniform of SplittableRandom(seed + state).
template <typename Src>
__global__ void __launch_bounds__(256) k_sample_shots(Src src_all, uint64_t len,
                                                      const double* prefix_all, uint64_t chunks,
                                                      const SampleScalars* sc,
                                                      const double* uniforms, uint64_t seed,
                                                      int64_t shots_per, int64_t shots_total,
                                                      int32_t* out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = warp; g < shots_total; g += nwarps) {
    const int64_t stn = g / shots_per;
    const int64_t k = g - stn * shots_per;
    const uint64_t off = (uint64_t)stn * len;
    auto src = [&](uint64_t i) { return src_all(off + i); };
    const double* prefix = prefix_all + (uint64_t)stn * chunks;
    const double scale = sc[stn].scale;
    const double u = uniforms ? uniforms[g] : splitmix_double(seed + (uint64_t)stn, (uint64_t)k);
    if (u >= 1.0) {
      if (lane == 0) out[g] = (int32_t)(len - 1);
      continue;
    }
    // last chunk whose prefix is < u (prefix[0] == 0)
    int64_t lo = 0, hi = (int64_t)chunks - 1, j = 0;
    while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (prefix[mid] < u) {
        j = mid;
        lo = mid + 1;
      } else {
        hi = mid - 1;
      }
    }
    const uint64_t b = (uint64_t)j * kChunk;
    constexpr int per = kChunk / 32;
    const uint64_t lb = b + (uint64_t)lane * per;
    double lsum = 0.0;
    for (int q = 0; q < per; ++q) {
      const uint64_t i = lb + q;
      if (i < len) lsum += src(i) * scale;
    }
    // exclusive warp scan of lane sums
    double incl = lsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    double run = prefix[j] + (incl - lsum);
    uint64_t found = ~0ULL;
    for (int q = 0; q < per; ++q) {
      const uint64_t i = lb + q;
      if (i >= len) break;
      run += src(i) * scale;
      if (i == len - 1 || run >= u) {  // the last entry is 1.0
        found = i;
        break;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t y = __shfl_xor_sync(0xffffffffu, found, o);
      found = y < found ? y : found;
    }
    if (lane == 0) {
      uint64_t r = found;
      if (r == ~0ULL) r = min(len - 1, b + kChunk);  // rounding gap: first entry of the next chunk
      out[g] = (int32_t)r;
    }
  }
}

// marginals: probs[o] = sum over the unmeasured bits r (ascending) of |a|^2
__device__ __forceinline__ uint64_t pdep64(uint64_t x, uint64_t mask) {
  uint64_t r = 0;
  for (uint64_t m = mask; m && x; m &= m - 1, x >>= 1)
    if (x & 1ULL) r |= m & (~m + 1ULL);
  return r;
}

template <typename R>
__global__ void k_marginal_seq(const typename Amp<R>::type* st, uint64_t mmask, uint64_t rmask,
                               uint64_t outcomes, uint64_t rest, double* probs) {
  DirectSrc<R> src{st};
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < outcomes;
       o += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t bo = pdep64(o, mmask);
    double acc = 0.0;
    for (uint64_t r = 0; r < rest; ++r) acc += src(bo | pdep64(r, rmask));
    probs[o] = acc;
  }
}

template <typename R>
__global__ void __launch_bounds__(kThreadsA)
    k_marginal_partial(const typename Amp<R>::type* st, uint64_t mmask, uint64_t rmask,
                       uint64_t outcomes, uint64_t rest, uint64_t chunks_per, double* partial) {
  __shared__ double red[kThreadsA / 32];
  DirectSrc<R> src{st};
  const uint64_t total = outcomes * chunks_per;
  for (uint64_t w = blockIdx.x; w < total; w += gridDim.x) {
    const uint64_t o = w / chunks_per, c = w % chunks_per;
    const uint64_t bo = pdep64(o, mmask);
    double acc = 0.0;
    for (int k = threadIdx.x; k < kChunk; k += kThreadsA) {
      const uint64_t r = c * kChunk + k;
      if (r < rest) acc += src(bo | pdep64(r, rmask));
    }
    const double s = block_sum<kThreadsA>(acc, red);
    if (threadIdx.x == 0) partial[w] = s;
  }
}

__global__ void k_marginal_final(const double* partial, uint64_t outcomes, uint64_t chunks_per,
                                 double* probs) {
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < outcomes;
       o += (uint64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (uint64_t c = 0; c < chunks_per; ++c) acc += partial[o * chunks_per + c];
    probs[o] = acc;
  }
}

int grid_cap(uint64_t work, int threads, int sm_count) {
  uint64_t b = (work + threads - 1) / threads;
  uint64_t cap = (uint64_t)sm_count * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

template <typename R>
cudaError_t marginal_t(const void* state, int n, uint64_t mmask, int m, double* probs,
                       double* scratch, size_t scratch_elems, int sm_count, cudaStream_t s) {
  const uint64_t outcomes = 1ULL << m;
  const uint64_t rest = 1ULL << (n - m);
  const uint64_t full = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
  const uint64_t rmask = full & ~mmask;
  auto st = static_cast<const typename Amp<R>::type*>(state);
  if (rest <= 64) {
    k_marginal_seq<R><<<grid_cap(outcomes, 256, sm_count), 256, 0, s>>>(st, mmask, rmask,
                                                                          outcomes, rest, probs);
  } else {
    const uint64_t chunks_per = (rest + kChunk - 1) / kChunk;
    if (outcomes * chunks_per > scratch_elems) return cudaErrorMemoryAllocation;
    k_marginal_partial<R><<<grid_cap(outcomes * chunks_per * kThreadsA, kThreadsA, sm_count),
                            kThreadsA, 0, s>>>(st, mmask, rmask, outcomes, rest, chunks_per,
                                               scratch);
    k_marginal_final<<<grid_cap(outcomes, 256, sm_count), 256, 0, s>>>(scratch, outcomes,
                                                                         chunks_per, probs);
  }
  return cudaGetLastError();
}

template <typename Src>
cudaError_t sample_src(Src src, uint64_t len, int64_t batch, const SampleArgs& a,
                       cudaStream_t s) {
  const uint64_t chunks = (len + kChunk - 1) / kChunk;
  const uint64_t all_chunks = chunks * (uint64_t)batch;
  k_chunk_sums<Src><<<grid_cap(all_chunks * kThreadsA, kThreadsA, a.sm_count), kThreadsA, 0, s>>>(
      src, len, chunks, a.chunk_sums, all_chunks);
  k_chunk_scan<<<(unsigned)batch, 1024, 0, s>>>(a.chunk_sums, chunks, a.chunk_prefix, a.scalars);
  if (a.shots > 0) {
    const int64_t total = a.shots * batch;
    const int blocks = grid_cap((uint64_t)total * 32, 256, a.sm_count);
    k_sample_shots<Src><<<blocks, 256, 0, s>>>(src, len, a.chunk_prefix, chunks, a.scalars,
                                               a.uniforms, a.seed, a.shots, total, a.outcomes);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_marginal(int dtype, const void* state, int n, uint64_t mmask, int m,
                            double* probs, double* scratch, size_t scratch_elems, int sm_count,
                            cudaStream_t s) {
  return dtype == SC_C64
             ? marginal_t<float>(state, n, mmask, m, probs, scratch, scratch_elems, sm_count, s)
             : marginal_t<double>(state, n, mmask, m, probs, scratch, scratch_elems, sm_count, s);
}

cudaError_t launch_sample(int dtype, const void* state, const double* probs, uint64_t len,
                          const SampleArgs& a, cudaStream_t s) {
  if (probs) return sample_src(ArraySrc{probs}, len, 1, a, s);
  if (dtype == SC_C64)
    return sample_src(DirectSrc<float>{static_cast<const float2*>(state)}, len, 1, a, s);
  return sample_src(DirectSrc<double>{static_cast<const double2*>(state)}, len, 1, a, s);
}

cudaError_t launch_sample_batch(int dtype, const void* states, uint64_t len, int64_t batch,
                                const SampleArgs& a, cudaStream_t s) {
  if (batch < 1 || batch > 65535) return cudaErrorInvalidValue;
  if (dtype == SC_C64)
    return sample_src(DirectSrc<float>{static_cast<const float2*>(states)}, len, batch, a, s);
  return sample_src(DirectSrc<double>{static_cast<const double2*>(states)}, len, batch, a, s);
}

uint64_t sample_chunks(uint64_t len) { return (len + kChunk - 1) / kChunk; }

}  // namespace sc
