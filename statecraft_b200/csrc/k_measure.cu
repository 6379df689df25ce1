// Measurement: marginal probabilities, the reference's running sum and per-shot search.
//
// Reference semantics (StatevectorEngine.java:229-338): probabilities over the
// measured qubits, rescaled by 1/sum when |sum - 1| > 1e-12 (the sum a left-to-right
// FP64 sum), a left-to-right FP64 running sum with the last entry forced to 1.0, and
// per shot the first index whose running sum is >= u (u >= 1 -> last index).
// Uniforms are the reference's SplittableRandom(seed).nextDouble() sequence,
// computed per shot from (seed, k).
//
// The running sum is reproduced bit for bit without a sequential pass over the whole
// array.  While a running sum S stays in one binade [2^e, 2^(e+1)), S is an integer A
// times ulp = 2^(e-52), and fl(S + p) = (A + round(p / ulp)) * ulp with round to
// nearest, ties to even (IEEE 754 round-to-nearest-even restated on integers): the
// result depends on A only through its parity, and only when p / ulp is exactly
// half-way.  A run of additions therefore acts on A as "add d0 if A is even, d1 if
// odd, and leave this parity", and such effects compose associatively.  Pass A sums
// chunks of kChunk probabilities approximately (FP64); pass B turns them into
// approximate running sums, which tell which chunks lie inside one binade (with a
// margin far above the summation error); pass C computes each such chunk's effect in
// integers (a chunk of zeros is the identity anywhere); pass D goes through the chunks
// in order from S = 0 -- runs of chunks in the running sum's binade as one scan of
// their effects, and the few chunks that cross a binade, start near zero or end the
// array by a warp that splits them the same way into 32 segments and adds one by one
// only inside the segments that cross -- and records the exact running sum before each
// chunk, the exact total and the rescaling decision; when the reference rescales,
// passes C and D run again on the rescaled probabilities (the running sums of pass B
// times the scale classify their chunks).  Pass E gives each shot a warp
// that binary-searches the exact chunk starts and replays its chunk: the exact start
// of each lane's segment (lane effects and a warp scan), then exact FP64 adds within
// each lane.
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

// pass A: sums[c] = sum of chunk c.  A batch of states of len_per entries each,
// stored back to back, has chunks_per chunks per state (chunk c of the whole array is
// chunk c % chunks_per of state c / chunks_per).
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

// pass B (one CTA of 1024 threads per state): approximate exclusive running sums of
// the chunk sums
__global__ void __launch_bounds__(1024) k_prefix_approx(const double* sums, uint64_t chunks,
                                                        double* prefix) {
  sums += blockIdx.x * chunks;
  prefix += blockIdx.x * chunks;
  __shared__ double part[1024];
  const uint64_t per = (chunks + 1023) / 1024;
  const uint64_t b = threadIdx.x * per;
  const uint64_t e = min(chunks, b + per);
  double local = 0.0;
  for (uint64_t c = b; c < e; ++c) local += sums[c];
  part[threadIdx.x] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0.0;
    for (int k = 0; k < 1024; ++k) {
      const double v = part[k];
      part[k] = run;
      run += v;
    }
  }
  __syncthreads();
  double run = part[threadIdx.x];
  for (uint64_t c = b; c < e; ++c) {
    prefix[c] = run;
    run += sums[c];
  }
}

// ---- integer form of the running sum inside one binade --------------------------
// ChunkTf::flags bits 2-4: an effect that holds in binade e; the effect applied (the
// chunk's start is the exact running sum and the chunk stays in binade e, or the chunk
// is all zeros); a chunk of zeros
constexpr int32_t kTfUsable = 4, kTfApplied = 8, kTfZero = 16;

// effect of a run of additions on A (the running sum in ulps of one binade)
struct Tf {
  int64_t d0, d1;  // increments for an even / odd A
  uint32_t p;      // bit 0: parity left for an even A, bit 1: for an odd A
};

__device__ __forceinline__ Tf tf_identity() { return Tf{0, 0, 2u}; }

// t1 then t2
__device__ __forceinline__ Tf tf_compose(const Tf& t1, const Tf& t2) {
  const uint32_t q0 = t1.p & 1u, q1 = (t1.p >> 1) & 1u;
  Tf r;
  r.d0 = t1.d0 + (q0 ? t2.d1 : t2.d0);
  r.d1 = t1.d1 + (q1 ? t2.d1 : t2.d0);
  r.p = ((t2.p >> q0) & 1u) | (((t2.p >> q1) & 1u) << 1);
  return r;
}

// the addition of p (>= 0) to a running sum in binade e, as an effect on A; *bad is
// set when p alone is too large to keep the sum in the binade
__device__ __forceinline__ Tf tf_of(double p, int e, bool* bad) {
  if (!(p > 0.0)) return tf_identity();
  const uint64_t bits = (uint64_t)__double_as_longlong(p);
  const int E = (int)((bits >> 52) & 0x7ffu);
  const uint64_t F = bits & ((1ULL << 52) - 1ULL);
  const uint64_t m = E ? (F | (1ULL << 52)) : F;
  const int q = E ? E - 1075 : -1074;  // p = m * 2^q
  const int s = q + 52 - e;            // p / ulp = m * 2^s
  uint64_t f;
  int cmp;  // fraction of p / ulp against one half: -1 below, 0 equal, 1 above
  if (s >= 0) {
    if (s > 9) {  // p / ulp >= 2^62: the sum leaves the binade
      *bad = true;
      return tf_identity();
    }
    f = m << s;
    cmp = -1;
  } else {
    const int t = -s;
    if (t >= 64) {
      f = 0;
      cmp = -1;  // m < 2^53 < 2^63: below one half
    } else {
      f = m >> t;
      const uint64_t rem = m & ((1ULL << t) - 1ULL);
      const uint64_t half = 1ULL << (t - 1);
      cmp = rem < half ? -1 : (rem == half ? 0 : 1);
    }
  }
  Tf r;
  if (cmp != 0) {
    const int64_t d = (int64_t)f + (cmp > 0 ? 1 : 0);
    r.d0 = r.d1 = d;
    const uint32_t dp = (uint32_t)(d & 1);
    r.p = dp | ((dp ^ 1u) << 1);
  } else {  // half-way: to the even neighbour, which leaves A even
    r.d0 = (int64_t)f + (int64_t)(f & 1ULL);
    r.d1 = (int64_t)f + (int64_t)((f + 1ULL) & 1ULL);
    r.p = 0u;
  }
  return r;
}

__device__ __forceinline__ Tf tf_shfl_up(const Tf& t, int o) {
  Tf r;
  r.d0 = __shfl_up_sync(0xffffffffu, t.d0, o);
  r.d1 = __shfl_up_sync(0xffffffffu, t.d1, o);
  r.p = __shfl_up_sync(0xffffffffu, t.p, o);
  return r;
}

// inclusive in-order scan of the lanes' effects
__device__ __forceinline__ Tf tf_warp_scan(Tf t, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const Tf u = tf_shfl_up(t, o);
    if (lane >= o) t = tf_compose(u, t);
  }
  return t;
}

// binade exponent of a positive normal double, or -2000 otherwise
__device__ __forceinline__ int binade(double s) {
  const uint64_t bits = (uint64_t)__double_as_longlong(s);
  const int E = (int)((bits >> 52) & 0x7ffu);
  return (E == 0 || E == 0x7ff || (bits >> 63)) ? -2000 : E - 1023;
}

// S = A * 2^(e - 52) with A in [2^52, 2^53): an effect applied to S, exactly; false
// when the result would leave the binade
__device__ __forceinline__ bool tf_apply(const Tf& t, int e, double* s) {
  const uint64_t bits = (uint64_t)__double_as_longlong(*s);
  const uint64_t A = (bits & ((1ULL << 52) - 1ULL)) | (1ULL << 52);
  const uint64_t An = A + (uint64_t)((A & 1ULL) ? t.d1 : t.d0);
  if (An >= (1ULL << 53)) return false;
  *s = __longlong_as_double((long long)(((uint64_t)(e + 1023) << 52) | (An - (1ULL << 52))));
  return true;
}

// The exact FP64 running sum over n <= 32 * PER values in order, from an exact start S,
// by one warp (every lane calls it; S uniform).  Lane l owns values [l PER, (l+1) PER)
// and gets back the exact running sum before its first value; *end gets the exact sum
// after all n.  Lanes whose segment stays inside one binade (approximate sums with a
// 2^-18 relative margin, far above their error) contribute integer effects; runs of
// such lanes in the binade of the running sum are one warp scan, and every other lane
// adds its values one by one from its exact start (in turn, so the work in sequence is
// the segments that cross a binade or start near zero).
template <int PER, typename Get>
__device__ double warp_exact_starts(const Get& get, uint32_t n, double S, int lane,
                                    double* end) {
  constexpr double kMargin = 0x1p-18;
  const uint32_t lb = (uint32_t)lane * PER;
  double a = 0.0;
  for (int q = 0; q < PER; ++q) {
    if (lb + q >= n) break;
    a += get(lb + q);
  }
  double incl = a;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const double ap_start = S + (incl - a), ap_end = S + incl;
  int e = binade(ap_start * (1.0 - kMargin));
  bool clean = e > -1000 && binade(ap_start) == e && binade(ap_end * (1.0 + kMargin)) == e;
  Tf t = tf_identity();
  if (clean) {
    bool bad = false;
    for (int q = 0; q < PER; ++q) {
      if (lb + q >= n) break;
      t = tf_compose(t, tf_of(get(lb + q), e, &bad));
    }
    clean = !bad;
  }
  double mine = S;
  // a run whose exact application fails (not expected under the margin) sends the
  // warp round again with every lane adding its own values
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (attempt == 1) clean = false;
    double Sx = S;  // exact running sum before lane L
    bool fail = false;
    for (int L = 0; L < 32;) {
      const int eL = __shfl_sync(0xffffffffu, e, L);
      const uint32_t ok = __ballot_sync(0xffffffffu, clean && e == eL && lane >= L);
      // lanes L .. D-1: one run of clean lanes in the binade of the running sum
      int D = L;
      if (binade(Sx) == eL) {
        const uint32_t rest = ~(ok >> L);
        D = rest ? L + __ffs(rest) - 1 : 32;
        if (D > 32) D = 32;
      }
      if (D > L) {
        const bool in = lane >= L && lane < D;
        const Tf ti = tf_warp_scan(in ? t : tf_identity(), lane);
        Tf te = tf_shfl_up(ti, 1);
        if (lane == 0) te = tf_identity();
        if (in) {
          double s = Sx;
          if (!tf_apply(te, eL, &s)) fail = true;
          mine = s;
        }
        double se = Sx;
        const bool ok_end = tf_apply(ti, eL, &se);
        Sx = __shfl_sync(0xffffffffu, se, D - 1);
        if (!__shfl_sync(0xffffffffu, ok_end, D - 1)) fail = true;
        L = D;
      }
      if (L < 32) {
        double s = Sx;
        if (lane == L) {
          mine = Sx;
          for (int q = 0; q < PER; ++q) {
            if (lb + q >= n) break;
            s = __dadd_rn(s, get(lb + q));
          }
        }
        Sx = __shfl_sync(0xffffffffu, s, L);
        ++L;
      }
    }
    if (!__any_sync(0xffffffffu, fail)) {
      *end = Sx;
      return mine;
    }
  }
  *end = S;  // not reached: the second attempt adds every value one by one
  return mine;
}

// pass C: per chunk, the binade its running sum stays in (from the approximate
// running sums, with a margin of 2^-18 relative, far above the summation error of at
// most 2^32 * 2^-53 relative) and its effect there.  One warp per chunk, in four
// sub-blocks of 512 values: a coalesced load into the warp's shared slab (padded one
// double per 16), then lane l takes the sub-block's values [16 l, 16 l + 16)
// (contiguous, so the lanes' effects compose in lane order), a warp scan, and the
// sub-block effects composed in order.  A chunk with no binade is checked for being
// all zeros.
constexpr int kSubBlock = 512;
constexpr int kSlab = kSubBlock + kSubBlock / 16;

template <typename Src>
__global__ void __launch_bounds__(kThreadsA) k_chunk_tf(Src src, uint64_t len_per,
                                                        uint64_t chunks_per, uint64_t chunks,
                                                        const double* prefix,
                                                        const SampleScalars* sc,
                                                        bool scaled_pass, ChunkTf* out) {
  constexpr double kMargin = 0x1p-18;
  constexpr int seg = kSubBlock / 32;
  __shared__ double slab_all[kThreadsA / 32][kSlab];
  const int lane = threadIdx.x & 31;
  double* const slab = slab_all[threadIdx.x >> 5];
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = warp0; c < chunks; c += nwarps) {
    const uint64_t st = c / chunks_per;
    if (scaled_pass && !sc[st].scaled) continue;
    const double scale = scaled_pass ? sc[st].scale : 1.0;
    const uint64_t cl = c - st * chunks_per;
    // clean: the whole chunk inside [2^e, 2^(e+1)) with the margin on both ends (the
    // last chunk, whose end is the total, is always added element by element).  On
    // the rescaled pass the running sums of the unscaled probabilities times the scale
    // stand in for those of the scaled ones (relative error ~2^-52 per value).
    int e = -2000;
    if (cl + 1 < chunks_per) {
      const double a = prefix[c] * scale, b = prefix[c + 1] * scale;
      const int ea = binade(a * (1.0 - kMargin));
      if (ea > -1000 && binade(a) == ea && binade(b * (1.0 + kMargin)) == ea) e = ea;
    }
    const uint64_t off = st * len_per;
    const uint64_t b0 = cl * kChunk;
    bool nz = false, bad = false;
    Tf total = tf_identity();
    for (int sb = 0; sb < kChunk / kSubBlock; ++sb) {
      const uint64_t base = b0 + (uint64_t)sb * kSubBlock;
      __syncwarp();  // the previous sub-block's reads of the slab are done
#pragma unroll
      for (int k = 0; k < seg; ++k) {
        const int q = k * 32 + lane;
        const uint64_t i = base + q;
        double pv = i < len_per ? src(off + i) : 0.0;
        if (scaled_pass) pv = __dmul_rn(pv, scale);
        slab[q + (q >> 4)] = pv;
      }
      __syncwarp();
      if (e < -1000) {
        // a chunk of zeros is the identity whatever the running sum (a sum of
        // values >= 0 is zero only when every value is)
#pragma unroll
        for (int k = 0; k < seg; ++k) nz = nz || slab[k * 32 + lane + ((k * 32 + lane) >> 4)] != 0.0;
        continue;
      }
      Tf t = tf_identity();
      const int q0 = lane * seg;
#pragma unroll
      for (int k = 0; k < seg; ++k) {
        const int q = q0 + k;
        t = tf_compose(t, tf_of(slab[q + (q >> 4)], e, &bad));
      }
      t = tf_warp_scan(t, lane);
      Tf sbt;  // the sub-block's effect, from lane 31
      sbt.d0 = __shfl_sync(0xffffffffu, t.d0, 31);
      sbt.d1 = __shfl_sync(0xffffffffu, t.d1, 31);
      sbt.p = __shfl_sync(0xffffffffu, t.p, 31);
      total = tf_compose(total, sbt);
    }
    if (e < -1000) {
      const bool any_nz = __any_sync(0xffffffffu, nz);
      if (lane == 0) out[c] = ChunkTf{0, 0, any_nz ? 0 : (2 | kTfZero), -2000};
      continue;
    }
    const bool any_bad = __any_sync(0xffffffffu, bad);
    if (lane == 0)
      out[c] = ChunkTf{total.d0, total.d1, (int32_t)(total.p & 3u) | (any_bad ? 0 : kTfUsable), e};
  }
}

// pass D (one CTA per state): the exact running sum before each chunk, in chunk
// order from S = 0; the exact total, the rescaling decision and the status.  On the
// rescaled pass, only the states the reference rescales.  Chunks go in blocks of
// 1024 records.  Within a block the CTA alternates two steps: the longest run of
// records from the current one whose effects hold in the binade of the running sum
// (chunks of zeros hold in any) is one in-order scan of their effects, each thread
// applying its exclusive prefix to the exact running sum; the record that ends the run
// is staged in shared memory by the CTA and added exactly by warp 0 (lane effects where
// they hold, one by one elsewhere).
template <typename Src>
__global__ void __launch_bounds__(1024) k_exact_starts(Src src, uint64_t len_per,
                                                       uint64_t chunks_per, ChunkTf* tfs,
                                                       double* starts, SampleScalars* sc,
                                                       bool scaled_pass) {
  const uint64_t st = blockIdx.x;
  if (scaled_pass && !sc[st].scaled) return;
  const double scale = scaled_pass ? sc[st].scale : 1.0;
  tfs += st * chunks_per;
  starts += st * chunks_per;
  const uint64_t off = st * len_per;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (int)(blockDim.x >> 5);
  __shared__ ChunkTf blk[1024];
  __shared__ double elems[kChunk];
  __shared__ Tf wsum[32];
  __shared__ uint32_t s_d;
  __shared__ double s_S;  // the exact running sum before record k
  if (threadIdx.x == 0) s_S = 0.0;
  for (uint64_t c0 = 0; c0 < chunks_per; c0 += 1024) {
    const uint32_t n_blk = (uint32_t)min((uint64_t)1024, chunks_per - c0);
    __syncthreads();
    if (threadIdx.x < n_blk) blk[threadIdx.x] = tfs[c0 + threadIdx.x];
    for (uint32_t k = 0; k < n_blk;) {
      if (threadIdx.x == 0) s_d = n_blk;
      __syncthreads();
      const double S = s_S;
      const int e = binade(S);
      const uint32_t i = threadIdx.x;
      bool zero = false, in = false;
      Tf t = tf_identity();
      if (i >= k && i < n_blk) {
        const ChunkTf& r = blk[i];
        zero = (r.flags & kTfZero) != 0;
        in = zero || ((r.flags & kTfUsable) && r.e == e && e > -1000);
        if (in && !zero) t = Tf{r.d0, r.d1, (uint32_t)(r.flags & 3)};
        if (!in) atomicMin(&s_d, i);
      }
      // in-order scan of the effects over the block (identity outside [k, n_blk))
      const Tf incl_w = tf_warp_scan(t, lane);
      if (lane == 31) wsum[warp] = incl_w;
      __syncthreads();
      const uint32_t D = s_d;
      if (warp == 0) {
        const Tf w = tf_warp_scan(lane < nwarps ? wsum[lane] : tf_identity(), lane);
        __syncwarp();
        wsum[lane] = w;  // inclusive over warps
      }
      __syncthreads();
      if (D > k) {
        Tf excl = tf_shfl_up(incl_w, 1);
        if (lane == 0) excl = tf_identity();
        if (warp > 0) excl = tf_compose(wsum[warp - 1], excl);
        const Tf incl = tf_compose(excl, t);
        // the run ends early where an effect does not keep the exact sum in the binade
        // (not expected: the records' binades carry a margin)
        double sv = S, se = S;
        bool ok_s = true, ok_e = true;
        if (e > -1000) {
          ok_s = tf_apply(excl, e, &sv);
          ok_e = tf_apply(incl, e, &se);
        }
        if (i >= k && i < D && !ok_e) atomicMin(&s_d, i);
        __syncthreads();
        const uint32_t D2 = s_d;
        if (i >= k && i < D2) {
          starts[c0 + i] = sv;
          blk[i].flags |= kTfApplied;
          (void)ok_s;
        }
        if (D2 > k && i == D2 - 1) s_S = se;
        __syncthreads();
        k = D2;
        if (k >= n_blk) break;
      }
      // record k: its chunk staged, then added exactly by warp 0
      const uint64_t b = (c0 + k) * kChunk;
      const uint32_t lim = (uint32_t)min((uint64_t)kChunk, len_per - b);
      for (uint32_t q = threadIdx.x; q < lim; q += blockDim.x) {
        double pv = src(off + b + q);
        if (scaled_pass) pv = __dmul_rn(pv, scale);
        elems[q] = pv;
      }
      __syncthreads();
      if (warp == 0) {
        const double S0 = s_S;
        double end = S0;
        warp_exact_starts<kChunk / 32>([&](uint32_t q) { return elems[q]; }, lim, S0, lane,
                                       &end);
        if (lane == 0) {
          starts[c0 + k] = S0;
          blk[k].flags &= ~kTfApplied;
          s_S = end;
        }
      }
      ++k;
    }
    __syncthreads();
    if (threadIdx.x < n_blk) tfs[c0 + threadIdx.x].flags = blk[threadIdx.x].flags;
  }
  __syncthreads();
  if (threadIdx.x == 0 && !scaled_pass) {
    // normalize (StatevectorEngine.java:298-312): a zero sum is an error; rescale by
    // 1.0 / sum when |sum - 1| > 1e-12
    const double S = s_S;
    sc[st].total = S;
    const bool zero = !(S > 0.0) || !isfinite(S);
    sc[st].status = zero ? 1 : 0;
    const bool rescale = !zero && fabs(S - 1.0) > 1e-12;
    sc[st].scaled = rescale ? 1 : 0;
    sc[st].scale = rescale ? __ddiv_rn(1.0, S) : 1.0;
  }
}

// pass E: one warp per shot.  In a batch, shot g belongs to state g / shots_per and
// draws the (g % shots_per)-th uniform of SplittableRandom(seed + state).
template <typename Src>
__global__ void __launch_bounds__(256) k_sample_shots(Src src_all, uint64_t len,
                                                      const double* starts_all,
                                                      const ChunkTf* tfs_all, uint64_t chunks,
                                                      const SampleScalars* sc,
                                                      const double* uniforms, uint64_t seed,
                                                      const uint64_t* seed_dev,
                                                      int64_t shots_per, int64_t shots_total,
                                                      int32_t* out) {
  const int lane = threadIdx.x & 31;
  if (seed_dev) seed = *seed_dev;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = warp; g < shots_total; g += nwarps) {
    const int64_t stn = g / shots_per;
    const int64_t k = g - stn * shots_per;
    const uint64_t off = (uint64_t)stn * len;
    const double* starts = starts_all + (uint64_t)stn * chunks;
    const ChunkTf* tfs = tfs_all + (uint64_t)stn * chunks;
    const bool scaled = sc[stn].scaled != 0;
    const double scale = sc[stn].scale;
    auto prob = [&](uint64_t i) {
      const double v = src_all(off + i);
      return scaled ? __dmul_rn(v, scale) : v;
    };
    const double u = uniforms ? uniforms[g] : splitmix_double(seed + (uint64_t)stn, (uint64_t)k);
    if (u >= 1.0) {
      if (lane == 0) out[g] = (int32_t)(len - 1);
      continue;
    }
    // last chunk whose exact start is < u (starts[0] == 0)
    int64_t lo = 0, hi = (int64_t)chunks - 1, j = 0;
    while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (starts[mid] < u) {
        j = mid;
        lo = mid + 1;
      } else {
        hi = mid - 1;
      }
    }
    const uint64_t b = (uint64_t)j * kChunk;
    const ChunkTf rec = tfs[j];
    constexpr int per = kChunk / 32;
    const uint64_t lb = b + (uint64_t)lane * per;
    // the exact running sum before this lane's values
    double run = starts[j];
    if ((rec.flags & kTfApplied) && !(rec.flags & kTfZero)) {
      // the chunk's sum stays in binade rec.e: the lanes' effects, scanned
      bool bad = false;
      Tf t = tf_identity();
      for (int q = 0; q < per; ++q) {
        const uint64_t i = lb + q;
        if (i >= len) break;
        t = tf_compose(t, tf_of(prob(i), rec.e, &bad));
      }
      const Tf incl = tf_warp_scan(t, lane);
      Tf excl = tf_shfl_up(incl, 1);
      if (lane == 0) excl = tf_identity();
      tf_apply(excl, rec.e, &run);
    } else if (!(rec.flags & kTfApplied)) {
      // a chunk that crosses a binade, starts near zero or ends the array
      double end;
      run = warp_exact_starts<per>([&](uint32_t q) { return prob(b + q); },
                                   (uint32_t)min((uint64_t)kChunk, len - b), run, lane, &end);
    }
    uint64_t found = ~0ULL;
    for (int q = 0; q < per; ++q) {
      const uint64_t i = lb + q;
      if (i >= len) break;
      run = __dadd_rn(run, prob(i));
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
      // not reached inside the chunk (the running sum at the chunk's end is >= u by
      // the search, so only a last-chunk tail below u): the last entry, forced to 1.0
      if (r == ~0ULL) r = min(len - 1, b + kChunk);
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
  const int grid_chunks = grid_cap(all_chunks * kThreadsA, kThreadsA, a.sm_count);
  const int grid_warps = grid_cap(all_chunks * 32, kThreadsA, a.sm_count);
  cudaError_t e = cudaMemsetAsync(a.scalars, 0, sizeof(SampleScalars) * (size_t)batch, s);
  if (e != cudaSuccess) return e;
  // the running sum of the probabilities, then (decided on the device, per state) of
  // the rescaled probabilities when the reference rescales
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 0) {
      k_chunk_sums<Src><<<grid_chunks, kThreadsA, 0, s>>>(src, len, chunks, a.chunk_sums,
                                                          all_chunks);
      k_prefix_approx<<<(unsigned)batch, 1024, 0, s>>>(a.chunk_sums, chunks, a.chunk_prefix);
    }
    k_chunk_tf<Src><<<grid_warps, kThreadsA, 0, s>>>(src, len, chunks, all_chunks,
                                                      a.chunk_prefix, a.scalars, pass == 1,
                                                      a.chunk_tf);
    k_exact_starts<Src><<<(unsigned)batch, 1024, 0, s>>>(src, len, chunks, a.chunk_tf,
                                                         a.chunk_start, a.scalars, pass == 1);
  }
  if (a.shots > 0) {
    const int64_t total = a.shots * batch;
    const int blocks = grid_cap((uint64_t)total * 32, 256, a.sm_count);
    k_sample_shots<Src><<<blocks, 256, 0, s>>>(src, len, a.chunk_start, a.chunk_tf, chunks,
                                               a.scalars, a.uniforms, a.seed, a.seed_dev, a.shots, total,
                                               a.outcomes);
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
