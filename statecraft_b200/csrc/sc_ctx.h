// The context behind the opaque sc_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "sc_internal.h"
#include "sc_measure.h"
#include "sc_noise.h"

namespace sc {

int fail(int code, const char* fmt, ...);
int fail_cuda(cudaError_t e, const char* where);
// frees a QAOA batch (sc_qaoa.cpp) and its device buffers
void qaoa_batch_free(void* batch);
// frees the cached trajectory batch (plans and CUDA graph, sc_trajectories.cpp)
void traj_cache_free(void* cache);
// context handle check (also makes its device current) and the op / noise-record
// validation of sc_run, shared with the batched entry points
int check_context(void* ctx);
int validate_circuit(int n, const sc_op* ops, int64_t n_ops, int max_qubits);
int validate_noise(const std::vector<sc_channel>& ch, const sc_op* ops, int64_t n_ops, int n);

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Ctx {
  static constexpr uint32_t kMagic = 0x5cb200u;
  uint32_t magic = kMagic;
  int device = 0;
  sc_config cfg{};
  cudaStream_t stream = nullptr;
  int sm_count = 148;
  int max_qubits = SC_DEFAULT_MAX_QUBITS;
  int low_qubits = 0;  // planner overrides (0 = default)
  int nr = 0;
  bool relayout = true;
  bool rotation = true;  // rotation form for 1-qubit unitaries in sweeps
  bool peephole = true;  // per-stage record peephole in the planner
  bool entry_fold = true;  // register permutations opening a stage folded into its read
  bool adjoint_fused = true;  // adjoint reverse pass as dual-state sweeps when it fits
  // runs of gates on <= 5 qubits whose sweep-path cost (FMA per amplitude) reaches this
  // become dense tensor-core blocks (complex128; 0 = never)
  double dense_block_cost = 160.0;

  // The plan of the last fused gate list (apply_sweeps), reused when the next run
  // plans the same gates on the same qubit count with the same settings: a circuit
  // simulated again (new seeds, new shots) skips the host planner.
  std::vector<PGate> plan_cache_gates;
  int plan_cache_n = -1;
  PlanParams plan_cache_pp{};
  Plan plan_cache;
  bool plan_cache_valid = false;

  // state
  int n = 0;
  DevBuf state;
  bool state_valid = false;
  std::vector<int32_t> default_measured;

  // noise schedule for the next run
  std::vector<sc_channel> noise;
  uint64_t noise_seed = 0;

  // device scratch (grow-only)
  size_t allocated = 0;
  DevBuf buf_err;                               // device error flag of bounded waits
  DevBuf buf_convert;                           // c64 <-> c128 staging
  DevBuf buf_noise_state, buf_noise_partial;    // Kraus trajectories
  DevBuf buf_sample;                            // chunk sums | prefix | scalars | uniforms | outcomes
  DevBuf buf_probs, buf_marg;                   // marginal probabilities
  DevBuf buf_expect;                            // Pauli partial sums
  DevBuf buf_adj_phi, buf_adj_lambda;           // adjoint work states
  DevBuf buf_traj_states, buf_traj_aux;         // trajectory batches: states | codes, sampling
  DevBuf buf_block;                             // dense block matrices of a run

  // adjoint bookkeeping
  std::vector<sc_op> adj_ops;
  std::vector<double> adj_params;
  std::vector<uint64_t> adj_x, adj_z;
  std::vector<double> adj_c;
  bool adj_ready = false;

  // QAOA batches created on this context (freed by sc_destroy)
  std::vector<void*> qaoa_batches;
  // the last trajectory batch: its plans and captured graph (freed by sc_destroy)
  void* traj_cache = nullptr;

  // plan statistics of the last run
  int64_t plan_sweeps_count = 0, plan_gates = 0, plan_stages = 0, plan_blocks = 0;

  // timing
  struct Timed {
    int cls;
    double bytes;
    cudaEvent_t a, b;
  };
  std::vector<Timed> pending;
  std::vector<cudaEvent_t> event_pool;
  size_t event_pool_next = 0;
  int64_t stats_launch[KC_COUNT] = {};
  double stats_ms[KC_COUNT] = {};
  double stats_bytes[KC_COUNT] = {};

  int reserve(DevBuf& b, size_t bytes, const char* what);
  void release(DevBuf& b);
  void release_all() {
    for (DevBuf* b : {&state, &buf_err, &buf_convert, &buf_noise_state,
                      &buf_noise_partial, &buf_sample, &buf_probs, &buf_marg, &buf_expect,
                      &buf_adj_phi, &buf_adj_lambda, &buf_traj_states, &buf_traj_aux,
                      &buf_block})
      release(*b);
  }
  void mark_begin(int cls, double bytes, int kernels = 1);
  void mark_end();
  cudaEvent_t get_event();
  void collect_timing();

  PlanParams plan_params() const;
  int ensure_state(int nq);
  int apply_gates(const std::vector<PGate>& gates);
  int apply_sweeps(const std::vector<PGate>& gates);
  int run(int nq, const sc_op* ops, int64_t n_ops, const double* init, uint64_t basis,
          bool has_basis, const double* params, int64_t n_params);
  int sample(const int32_t* qubits, int32_t m, int64_t shots, uint64_t seed,
             const double* uniforms, int32_t* outcomes);
  int probabilities(const int32_t* qubits, int32_t m, double* out);
  int pauli_terms(int32_t n_terms, const uint64_t* xmask, const uint64_t* zmask,
                  std::vector<double>& terms);
};

}  // namespace sc
