// Measurement launchers (k_measure.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

constexpr int kSampleChunk = 2048;  // probabilities per chunk of the two-level prefix sum

struct SampleScalars {
  double total;  // sum of the probabilities
  double scale;  // 1/total when |total - 1| > 1e-12, else 1
  int32_t status;  // 1: zero or non-finite total
  int32_t pad;
};

struct SampleArgs {
  double* chunk_sums;    // device, sample_chunks(len) doubles
  double* chunk_prefix;  // device, sample_chunks(len) doubles
  SampleScalars* scalars;  // device
  const double* uniforms;  // device or nullptr (then SplitMix64(seed))
  uint64_t seed;
  int64_t shots;         // 0: only the prefix sums
  int32_t* outcomes;     // device, shots entries
  int sm_count;
};

uint64_t sample_chunks(uint64_t len);

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
