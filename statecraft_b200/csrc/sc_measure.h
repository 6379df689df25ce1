// Measurement launchers (k_measure.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

constexpr int kSampleChunk = 2048;  // probabilities per chunk of the two-level prefix sum

struct SampleScalars {
  double total;  // the reference's left-to-right sum of the probabilities (exact)
  double scale;  // 1/total when |total - 1| > 1e-12, else 1
  int32_t status;  // 1: zero or non-finite total
  int32_t scaled;  // 1: the probabilities are rescaled by `scale` before the running sum
};

// Per-chunk record of the exact running sum (k_measure.cu): the effect of the chunk's
// additions on a running sum that stays in one binade [2^e, 2^(e+1)), as integer
// increments in units of that binade's ulp for an even (d0) and an odd (d1) running
// sum, and the parity it leaves (flags bit 0: for an even sum, bit 1: for an odd
// one); flags bit 2: usable (the chunk lies in one binade and the record was
// computed); bit 3: set by the exact pass when the record was applied (else the
// chunk was added element by element).
struct ChunkTf {
  int64_t d0, d1;
  int32_t flags;
  int32_t e;
};

struct SampleArgs {
  double* chunk_sums;    // device, sample_chunks(len) doubles per state
  double* chunk_prefix;  // device, the same: approximate running sums before each chunk
  double* chunk_start;   // device, the same: exact running sums before each chunk
  ChunkTf* chunk_tf;     // device, sample_chunks(len) records per state
  SampleScalars* scalars;  // device, one per state
  const double* uniforms;  // device or nullptr (then SplitMix64(seed))
  uint64_t seed;
  const uint64_t* seed_dev = nullptr;  // device copy of the seed, read instead of `seed`
  int64_t shots;         // 0: only the prefix sums
  int32_t* outcomes;     // device, shots entries
  int sm_count;
};

uint64_t sample_chunks(uint64_t len);
// kernels one launch_sample / launch_sample_batch enqueues (chunk sums, running sums,
// chunk effects and exact starts; effects and exact starts again for the rescaled
// probabilities; the per-shot search)
constexpr int kSampleKernels = 7;

// probs[o] = marginal probability of outcome o over the measured mask (m bits).
// scratch must hold 2^m * ceil(2^(n-m) / kSampleChunk) doubles when 2^(n-m) > 64.
cudaError_t launch_marginal(int dtype, const void* state, int n, uint64_t mmask, int m,
                            double* probs, double* scratch, size_t scratch_elems, int sm_count,
                            cudaStream_t s);

// Samples from |amp_i|^2 (probs == nullptr) or from probs[0..len).
cudaError_t launch_sample(int dtype, const void* state, const double* probs, uint64_t len,
                          const SampleArgs& a, cudaStream_t s);

// A batch of `batch` states of len amplitudes each, back to back: chunk sums /
// prefixes / scalars per state (batch * sample_chunks(len), batch entries),
// a.shots shots per state, state b drawing from SplittableRandom(a.seed + b);
// outcomes[b * a.shots + k].
cudaError_t launch_sample_batch(int dtype, const void* states, uint64_t len, int64_t batch,
                                const SampleArgs& a, cudaStream_t s);

}  // namespace sc
