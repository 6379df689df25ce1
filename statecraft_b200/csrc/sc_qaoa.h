// Batched QAOA ring ansatz: device records and launchers (k_qaoa.cu), used by
// the batch object in sc_qaoa.cpp.
//
// Instance i has n_i qubits and p layers (gamma_l, beta_l).  Its circuit is H on
// every qubit, then per layer the ring cost phase prod_j exp(-i gamma_l Z_j Z_{j+1 mod n})
// and RX(2 beta_l) on every qubit (app/.../AlgorithmSuiteSpecs.java:186-200,
// 283-296); the output is <sum_j Z_j Z_{j+1 mod n}> in FP64.
//
// The cost phase of basis state x is exp(-i gamma (n - 2 k(x))) with
// k(x) = popcount(x XOR rotr_n(x)), so a layer's n two-qubit diagonals are one
// table lookup of n + 1 precomputed phases per amplitude.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

constexpr int kQaoaTileQubits = 12;  // qubits of a shared-memory tile
constexpr int kQaoaMaxQubits = 23;   // high passes need n - 12 < 12
constexpr int kQaoaMaxLayers = 16;

enum QaoaMode : int32_t {
  kQaoaWhole = 0,  // n <= 12: the whole instance lives in one CTA's shared memory
  kQaoaLow = 1,    // tile = qubits 0..11 (contiguous 4096 amplitudes)
  kQaoaHigh = 2,   // tile = qubits 12..n-1 plus the 24 - n lowest (contiguous runs)
};

struct QaoaInst {
  int32_t n;        // qubits
  int32_t orig;     // index in the caller's instance order
  int64_t amp_off;  // offset of the state in the arena (amplitudes); whole mode: unused
  int64_t ph_off;   // offset of the phase tables (complex entries): layer l at + l * (n + 1)
};

// One pass over the large instances: RX(layer rx_a) on the tile's gate qubits,
// the cost phase of layer d, RX(layer rx_b); -1 skips a step.  init: the state
// starts as H^n |0>; reduce: accumulate the energy instead of storing.
struct QaoaPass {
  int32_t mode;
  int32_t init;
  int32_t rx_a, d, rx_b;
  int32_t reduce;
};

struct QaoaLaunch {
  void* state;                 // arena (double2 / float2)
  const QaoaInst* inst;        // this launch's instance list
  const int64_t* item_prefix;  // n_inst + 1 item offsets
  int32_t n_inst;
  int32_t p;
  int64_t n_items;
  const double* cs;            // RX (t, form) at 2 * (orig * p + l), see sc_qaoa.cpp
  const double* escale;        // per instance: energy / norm factor of the last RX scalars
  const double* phase;         // (re, im) pairs
  double* partials;            // (energy, norm) per item
  int64_t part_base;           // partial slot of item 0
};

// partial slots of instance orig: [begin, end)
struct QaoaSpan {
  int64_t begin, end;
};

// Kernel shapes the autotuner chooses from (register qubits per thread, CTAs per
// SM the register budget is sized for, double-buffered tiles):
// 0 = 4,2,no  1 = 4,2,yes  2 = 3,1,no  3 = 3,2,yes
constexpr int kQaoaShapes = 4;
int qaoa_shape_nr(int shape);
cudaError_t launch_qaoa(int dtype, int shape, const QaoaLaunch& a, const QaoaPass& pass,
                        int ctas_per_sm, int sm_count, cudaStream_t s);
cudaError_t launch_qaoa_reduce(const double* partials, const QaoaSpan* spans, int64_t n_inst,
                               double* energies, double* norms, cudaStream_t s);
// largest ctas_per_sm the kernel shape can keep resident (0 on error)
int qaoa_max_ctas_per_sm(int dtype, int shape, int p);

}  // namespace sc
