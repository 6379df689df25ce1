// Adjoint-differentiation launchers (k_adjoint.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

int adjoint_partial_blocks(int n, int sm_count);

// out = sum_k c_k P_k psi (terms applied up to 64 per pass, FP64 sums)
cudaError_t launch_pauli_sum(int dtype, const void* psi, void* out, int n, const uint64_t* x,
                             const uint64_t* z, const double* c, int64_t count, int sm_count,
                             cudaStream_t s);
// partial[block] = the block's share of <lam | psi> (adjoint_partial_blocks blocks)
cudaError_t launch_inner(int dtype, const void* lam, const void* psi, int n, double2* partial,
                         int sm_count, cudaStream_t s);
// grad[slot] += Im <lam | P | psi>, P = i^{|x&z|} X^x Z^z
cudaError_t launch_generator_grad(int dtype, const void* lam, const void* psi, int n, uint64_t x,
                                  uint64_t z, double2* partial, double* grad, int slot,
                                  int sm_count, cudaStream_t s);

}  // namespace sc
