// Kraus trajectory launchers (k_noise.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/statecraft_b200.h"

namespace sc {

struct KrausArgs {
  double k[SC_MAX_KRAUS][8];
  int32_t nk;
  int32_t target;
};

constexpr int kNoiseBadWeight = 1;  // a branch weight is negative or not finite
constexpr int kNoiseBadTotal = 2;   // total weight not finite or <= 1e-15
constexpr int kNoiseBadNorm = 3;    // state norm zero / not finite after the Kraus operator
constexpr int kNoiseChoiceRing = 4096;

// Device-resident trajectory bookkeeping (one per context).
struct NoiseDevState {
  int32_t status;       // 0 or kNoiseBad*
  int32_t last_choice;
  uint64_t bad_draw;
  double matrix[8];     // chosen K / sqrt(w)
  int32_t choices[kNoiseChoiceRing];  // chosen index per draw (mod ring)
};

int noise_grid(int n, int sm_count);

// Weights sweep + select + apply for one (channel, target).  `partial` holds
// noise_grid(n) * SC_MAX_KRAUS doubles.  `draw` is the index of this draw in the
// noise stream (the d-th rng.nextDouble(total) of SplittableRandom(seed)).
cudaError_t launch_kraus_channel(int dtype, void* state, int n, const KrausArgs& a,
                                 uint64_t seed, uint64_t draw, double* partial,
                                 NoiseDevState* ns, int sm_count, cudaStream_t s);

// Weights and draw of one Kraus point for `batch` states of n qubits stored back to
// back (trajectory t draws from SplittableRandom(seeds[0] + t), seeds in device
// memory).  K_k / sqrt(w_k) of state t goes to mats + t * 8 (reals of the dtype) for
// the next sweep to apply; with `pend`, state t's matrix pend + t * 8 on qubit pend_q
// (not yet applied) is applied before weighing.  partial holds batch *
// noise_grid_batch(n, batch) * SC_MAX_KRAUS doubles; the chosen index of state t goes
// to choices[t * choice_stride]; a state whose status is nonzero is skipped, and a
// failed draw sets it (kNoiseBad*).
int noise_grid_batch(int n, int64_t batch, int sm_count);
cudaError_t launch_kraus_batch(int dtype, const void* states, int n, int64_t batch,
                               const KrausArgs& a, int pend_q, const void* pend,
                               const uint64_t* seeds, uint64_t draw, double* partial, void* mats,
                               int32_t* choices, int64_t choice_stride, int32_t* status,
                               int sm_count, cudaStream_t s);

// Pauli-sum expectation: out_partial[t] receives term t's <psi|P_t|psi> (real part).
cudaError_t launch_pauli_terms(int dtype, const void* state, int n, int n_terms,
                               const uint64_t* xmask, const uint64_t* zmask, double* partial,
                               size_t partial_elems, double* out_terms, int sm_count,
                               cudaStream_t s);
int pauli_partial_cols(int n, int sm_count);

}  // namespace sc
