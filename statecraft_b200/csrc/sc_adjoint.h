// Adjoint-differentiation launchers (k_adjoint.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

int adjoint_partial_blocks(int n, int sm_count);

// out = c * P psi (accumulate = false) or out += c * P psi
cudaError_t launch_pauli_accumulate(int dtype, const void* psi, void* out, int n, uint64_t x,
                                    uint64_t z, double c, bool accumulate, int sm_count,
                                    cudaStream_t s);

// grad[slot] += Im <lam | P | psi>, P = i^{|x&z|} X^x Z^z
cudaError_t launch_generator_grad(int dtype, const void* lam, const void* psi, int n, uint64_t x,
                                  uint64_t z, double2* partial, double* grad, int slot,
                                  int sm_count, cudaStream_t s);

}  // namespace sc
