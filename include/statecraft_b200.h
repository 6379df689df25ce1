/*
 * statecraft_b200.h -- C ABI of the B200-native dense statevector engine.
 *
 * This is the drop-in boundary for StateCraft's `statevector` engine hot path.
 * A host engine class (Java FFM downcalls, Python ctypes, C/C++) walks
 * QuantumCircuit.operations(), flattens them into an array of `sc_op`, and calls
 * these entry points.  Plain C types only: pointers, sizes, POD structs.
 *
 * Conventions
 *   - Every entry point returns SC_OK (0) or a negative status.  The message of
 *     the last failure on the calling thread is returned by sc_last_error().
 *     Status -> reference exception mapping (StatevectorEngine.java):
 *        SC_EINVAL        IllegalArgumentException      (bad qubit, bad noise target)
 *        SC_EUNSUPPORTED  UnsupportedOperationException (unitary after measure, size limit)
 *        SC_ESTATE        IllegalStateException         (zero norm, invalid Kraus weights)
 *        SC_ENOMEM / SC_ECUDA / SC_ETIMEOUT             device-side failures
 *   - All host buffers are caller-owned; the library keeps no pointer past return.
 *   - Device memory is owned by the context.  A context is single-threaded
 *     (one CUDA stream); callers serialise calls on one context.
 *   - Amplitudes cross the boundary as interleaved doubles [re0, im0, re1, ...]
 *     with little-endian qubit order (qubit q is bit q of the basis index), the
 *     layout of core/.../quantum/StateVector.java.
 */
#ifndef STATECRAFT_B200_H
#define STATECRAFT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_ABI_VERSION 2

#if defined(__GNUC__)
#define SC_API __attribute__((visibility("default")))
#else
#define SC_API
#endif

/* ---- status codes ------------------------------------------------------ */
#define SC_OK 0
#define SC_EINVAL (-1)
#define SC_EUNSUPPORTED (-2)
#define SC_ESTATE (-3)
#define SC_ENOMEM (-4)
#define SC_ECUDA (-5)
#define SC_ETIMEOUT (-6)

/* ---- amplitude storage types ------------------------------------------- */
#define SC_C128 0 /* complex128: the drop-in; matches the Java double[] engine */
#define SC_C64 1  /* complex64 bulk; FP64 kept for norms, reductions, CDF, inner products */

/* ---- operation kinds (QuantumCircuit.Operation, QuantumCircuit.java:362-574) */
#define SC_OP_SINGLE 1  /* SingleGateOperation: q0 = target, m[0..7] = 2x2 row-major complex */
#define SC_OP_CNOT 2    /* CnotOperation: q0 = control, q1 = target */
#define SC_OP_TWO 3     /* TwoQubitGateOperation: q0 = first, q1 = second, m[0..31] = 4x4
                           row-major complex; local basis index = 2*bit(first) + bit(second) */
#define SC_OP_DIAG2 4   /* TwoQubitDiagonalOperation: q0 = first, q1 = second, m[0..7] = d[4] */
#define SC_OP_SWAP 5    /* SwapOperation: q0, q1 */
#define SC_OP_MULTI 6   /* MultiControlOperation: q0 = target, mask = control qubits,
                           m[0..7] = 2x2 gate */
#define SC_OP_MEASURE 7 /* MeasureOperation: mask = measured qubits */
/* Parameterised rotations (adjoint-gradient and batched additions).  The angle is
 * params[param] when param >= 0 and a parameter vector is supplied, else m[0].
 * Conventions of core/.../parse/OpenQasmCircuitParser.java:650-670. */
#define SC_OP_RX 16  /* exp(-i a/2 X) on q0 */
#define SC_OP_RY 17  /* exp(-i a/2 Y) on q0 */
#define SC_OP_RZ 18  /* exp(-i a/2 Z) on q0 */
#define SC_OP_RZZ 19 /* exp(-i a/2 Z(q0) Z(q1)) */

typedef struct sc_op {
  int32_t kind;  /* SC_OP_* */
  int32_t q0;    /* see the kind */
  int32_t q1;    /* see the kind; -1 when unused */
  int32_t param; /* parameter index for SC_OP_R*, else -1 */
  uint64_t mask; /* control mask (SC_OP_MULTI) or measured mask (SC_OP_MEASURE) */
  double m[32];  /* matrix / diagonal entries as (re, im) pairs */
} sc_op;

/* One scheduled application of a single-qubit Kraus channel, flattened from
 * NoiseModel.scheduledChannelsAfter(op) (NoiseModel.java:211-241): the host
 * resolves composite channels and mapped targets and emits one record per
 * (channel, target) in the order StatevectorEngine.applyErrorChannel visits them
 * (StatevectorEngine.java:382-407).  Records must be sorted by after_op. */
#define SC_MAX_KRAUS 8
typedef struct sc_channel {
  int64_t after_op; /* index into the op array of the operation this follows */
  int32_t target;   /* qubit */
  int32_t n_kraus;  /* 1..SC_MAX_KRAUS */
  double kraus[SC_MAX_KRAUS][8]; /* each a 2x2 row-major complex matrix */
} sc_channel;

typedef struct sc_config {
  int32_t dtype;            /* SC_C128 (default) or SC_C64 */
  int32_t fusion;           /* 1 = fused tile sweeps (default), 0 = one kernel per gate */
  int32_t tile_qubits;      /* qubits per shared-memory tile; 0 = default */
  int32_t sweep_budget;     /* FP FMA per amplitude allowed per sweep; 0 = default, <0 = unlimited */
  int32_t max_qubits;       /* dense limit; 0 = default (SC_DEFAULT_MAX_QUBITS) */
  int32_t timing;           /* 1 = record CUDA-event time per kernel class */
  int64_t device_mem_limit; /* bytes of device memory the context may allocate; 0 = no cap.
                               Exceeding it returns SC_ENOMEM without calling the allocator. */
  int32_t autotune;         /* 1 = sc_trajectories times a few tile shapes on the first batch
                               of a circuit and keeps the fastest (0 = the configured shape) */
  int32_t reserved;
} sc_config;

#define SC_DEFAULT_MAX_QUBITS 32

/* ---- library / context --------------------------------------------------- */
SC_API int32_t sc_version(void);
SC_API const char* sc_last_error(void);
/* Replaces `new StatevectorEngine(StatevectorExecutionConfig)` (StatevectorEngine.java:46-55). */
SC_API int32_t sc_create(int32_t device, const sc_config* cfg, void** out_ctx);
SC_API int32_t sc_destroy(void* ctx);

/* ---- simulate ------------------------------------------------------------- */
/* Noise schedule for the next sc_run (StatevectorEngine.java:79-85, 371-600).
 * It is consumed by that run (one schedule per run); n = 0 clears it.
 * has_seed = 0 draws a fresh seed, like `new SplittableRandom()`. */
SC_API int32_t sc_set_noise(void* ctx, const sc_channel* channels, int64_t n, uint64_t seed,
                     int32_t has_seed);

/* Replaces the state preparation and op loop of StatevectorEngine.simulate
 * (StatevectorEngine.java:63-151).  init_state (nullable) holds 2^(n+1) doubles
 * (populateFromState); else has_basis selects resetBasisState(basis_mask); else |0..0>. */
SC_API int32_t sc_run(void* ctx, int32_t n_qubits, const sc_op* ops, int64_t n_ops,
               const double* init_state, uint64_t basis_mask, int32_t has_basis);

/* Copies the final state out as interleaved doubles (StatevectorEngine.java:153-155). */
SC_API int32_t sc_get_state(void* ctx, double* out, int64_t n_doubles);

/* Measured qubits resolved like resolveMeasuredQubits (StatevectorEngine.java:259-272):
 * the qubits of the MeasureOperations of the last run, sorted and distinct, else all.
 * Returns the count (>= 0) and writes up to cap entries. */
SC_API int32_t sc_default_measured_qubits(void* ctx, int32_t* out, int32_t cap);

/* Replaces performMeasurement + sampleOutcome (StatevectorEngine.java:229-257, 274-338).
 * qubits: ascending distinct measured qubits (m >= 1).  Outcome bit k <-> qubits[k].
 * Uniform draws: uniforms[shot] when non-null, else SplittableRandom(seed).nextDouble()
 * per shot (has_seed = 0: a fresh random seed).  outcomes: caller-owned int32[shots]. */
SC_API int32_t sc_sample(void* ctx, const int32_t* qubits, int32_t m, int64_t shots, uint64_t seed,
                  int32_t has_seed, const double* uniforms, int32_t* outcomes);

/* Normalised marginal probabilities over the measured qubits (the array that
 * StatevectorEngine.computeMeasurementProbabilities + normalize produce,
 * StatevectorEngine.java:274-312).  out: caller-owned double[2^m]. */
SC_API int32_t sc_probabilities(void* ctx, const int32_t* qubits, int32_t m, double* out);

/* ---- additions (no counterpart in the reference engine) -------------------- */
/* <psi| sum_k c_k P_k |psi> on the current state; P_k = prod X^x Z^z with Y = iXZ,
 * i.e. term k acts as X on bits of xmask[k], Z on bits of zmask[k], Y on both. */
SC_API int32_t sc_expect_pauli(void* ctx, int32_t n_terms, const uint64_t* xmask,
                        const uint64_t* zmask, const double* coeffs, double* out_value);

/* Adjoint differentiation: forward runs the parameterised circuit from |0..0>
 * and evaluates <H>; backward returns dE/dparams in one reverse sweep with two
 * state buffers and no stored intermediate states. */
SC_API int32_t sc_adjoint_forward(void* ctx, int32_t n_qubits, const sc_op* ops, int64_t n_ops,
                           const double* params, int64_t n_params, int32_t n_terms,
                           const uint64_t* xmask, const uint64_t* zmask, const double* coeffs,
                           double* out_value);
SC_API int32_t sc_adjoint_backward(void* ctx, double* out_grad, int64_t n_params);

/* Batched QAOA ring ansatz (no counterpart in the reference engine, which runs
 * such suites one circuit at a time through simulate(); the ansatz is
 * app/.../AlgorithmSuiteSpecs.java:186-200, phases :283-287).  Instance i has
 * n_qubits[i] in 2..23 qubits; its circuit is H on every qubit, then for each of
 * the p (1..16) layers exp(-i gammas[i*p+l] Z_j Z_{j+1 mod n}) on every ring edge
 * and RX(2 betas[i*p+l]) on every qubit; the result is <sum_j Z_j Z_{j+1 mod n}>.
 * All instances run in one captured CUDA graph of p + 3 kernels over uneven
 * instance sizes; dtype SC_C64 keeps amplitudes in complex64 and every table and
 * reduction in FP64.  tune = 1 times the kernel shapes on the batch and keeps the
 * fastest.  States of instances with more than 12 qubits live in one device arena
 * (2^n amplitudes each); smaller ones never leave shared memory.
 * A batch belongs to its context (freed with it at the latest). */
SC_API int32_t sc_qaoa_batch_create(void* ctx, int32_t dtype, int64_t n_inst, const int32_t* n_qubits,
                                    int32_t p, const double* gammas, const double* betas,
                                    int32_t tune, void** out_batch);
/* New angles for the next runs (same shapes; the captured graph is reused). */
SC_API int32_t sc_qaoa_batch_set_angles(void* batch, const double* gammas, const double* betas);
/* Enqueues one run of the whole batch (one graph launch) on the context stream. */
SC_API int32_t sc_qaoa_batch_run(void* batch);
/* Waits for the runs and copies <sum ZZ> (and the FP64 norms) per instance, in
 * the caller's instance order; either pointer may be NULL. */
SC_API int32_t sc_qaoa_batch_energies(void* batch, double* energies, double* norms);
/* Chosen shape (register group width, CTAs per SM), its tuned time per run and
 * the algorithmic HBM bytes per run. */
SC_API int32_t sc_qaoa_batch_info(void* batch, int32_t* nr, int32_t* ctas_per_sm, double* tuned_ms,
                                  double* bytes_per_run);
SC_API int32_t sc_qaoa_batch_destroy(void* batch);

/* Batched noisy trajectories (no counterpart in the reference engine, which runs
 * one trajectory per simulate(); trajectory semantics StatevectorEngine.java:371-600).
 * Runs n_traj (1..65535) copies of the circuit from |0..0> in the context's dtype;
 * trajectory t draws its Kraus branches from SplittableRandom(noise_seed + t), one
 * nextDouble(total) per noise record in record order, and samples `shots` outcomes
 * of all qubits from SplittableRandom(measure_seed + t).  Records that are Pauli
 * mixtures (each Kraus operator a scalar times I, X, Y or Z: depolarizing, bit flip,
 * phase flip, ...) have state-independent weights: their branches are drawn on the
 * host and applied inside the fused sweeps.  Any other record (amplitude or phase
 * damping, thermal relaxation, ...) ends a fused segment: its branch weights
 * ||K_k psi||^2 are summed on the device for every trajectory, the branch drawn
 * there and K_k / sqrt(w_k) applied.  Invalid weights return SC_ESTATE (the
 * reference's IllegalStateException).  Records are sc_channel, sorted by after_op,
 * e.g. one per touched qubit after each gate.  Outputs (caller-owned, any may be
 * NULL): outcomes[t*shots + k] (basis index), choices[t*n_channels + j] (chosen Kraus
 * index), states[t * 2^(n+1) ...] (interleaved doubles of every final state; small
 * batches only).  The context keeps the plans of its last batch and, unless
 * cfg.timing is set, a CUDA graph of the batch's device work: a later call with the
 * same circuit, records, n_traj, shots and configuration replays the graph (only the
 * branch table and the seeds are uploaded). */
SC_API int32_t sc_trajectories(void* ctx, int32_t n_qubits, const sc_op* ops, int64_t n_ops,
                               const sc_channel* channels, int64_t n_channels, int64_t n_traj,
                               uint64_t noise_seed, int64_t shots, uint64_t measure_seed,
                               int32_t* outcomes, int32_t* choices, double* states);
/* The last trajectory batch of the context: tile qubits and register qubits it was
 * planned with, 1 if a CUDA graph of it is held, and the time (ms) of the fastest
 * shape when cfg.autotune chose it (0 otherwise).  Any pointer may be NULL. */
SC_API int32_t sc_trajectories_info(void* ctx, int32_t* tile_qubits, int32_t* nr, int32_t* graph,
                                    double* tuned_ms);

/* Per-kernel-class device timing collected while cfg.timing = 1:
 * for class i in [0, cap): launches[i], milliseconds[i], bytes[i] (algorithmic
 * bytes moved).  Returns the number of classes; names via sc_kernel_class_name. */
SC_API int32_t sc_kernel_stats(void* ctx, int64_t* launches, double* milliseconds, double* bytes,
                        int32_t cap);
SC_API const char* sc_kernel_class_name(int32_t cls);
SC_API int32_t sc_reset_kernel_stats(void* ctx);

/* The context's CUDA stream (a cudaStream_t), so callers can time its work with
 * their own CUDA events. */
SC_API void* sc_stream(void* ctx);

/* Plan statistics of the last sc_run: sweeps launched, gates, stages. */
SC_API int32_t sc_last_plan_stats(void* ctx, int64_t* sweeps, int64_t* gates, int64_t* stages);

/* Sampling that allocates nothing.  No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc when they sample -- frameworks whose device
 * memory belongs to their own pool allocator, serving loops that must not allocate
 * after start-up, and processes that have already handed the GPU's memory to their
 * own buffers.  Samples every qubit of a state the caller holds in device memory
 * (d_state: 2^n amplitudes of `dtype`; outcome = basis index) into the caller's
 * device buffer d_outcomes[shots], on the caller's cudaStream_t `stream`, and
 * returns after the stream has finished (on a stream that is capturing it returns
 * SC_EINVAL and enqueues nothing).
 * Uniforms: d_uniforms[shot] (device, nullable) else SplittableRandom(seed).
 * Scratch is a fixed array in the library's device data sized for at most 2^30
 * amplitudes (30 qubits, about 24 MiB held by every GPU that loads the library);
 * larger states return SC_EINVAL.  The first call on a device looks the array up
 * (make it before any stream capture); a cudaDeviceReset after that is not
 * supported.  All calls share the array: calls that overlap on the GPU race. */
SC_API int32_t sc_sample_static(const void* d_state, int32_t n_qubits, int32_t dtype,
                                int64_t shots, uint64_t seed, const double* d_uniforms,
                                int32_t* d_outcomes, void* stream);

/* ---- host-only planner inspection (no GPU needed; used by the test suite) --- */
/* Op indices in the order the fused sweeps apply them; returns the gate count.
 * Also reports the number of sweeps, stages, sweeps that change the qubit layout
 * and layout-restoring permutation passes (any out pointer may be NULL). */
SC_API int32_t sc_debug_plan_order(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                            int32_t low_qubits, int32_t nr, double budget, int64_t* order,
                            int64_t* n_sweeps, int64_t* n_stages, int64_t* n_relayouts,
                            int64_t* n_restores);
/* Entry folds of the plan of ops: stats[3] = {stages, records folded into a stage's
 * read (register permutations opening a stage), of which conditional (an X with
 * controls outside the registers, applied as a per-thread read flip)}. */
SC_API int32_t sc_debug_entry_folds(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                                    int32_t low_qubits, int32_t nr, double budget, int64_t* stats);
/* Executes the sweep plan on a host complex128 state (interleaved doubles) with the
 * kernel's tile / stage / register semantics; returns the number of sweeps. */
SC_API int32_t sc_debug_emulate_sweeps(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                                int32_t low_qubits, int32_t nr, double budget, double* state);
/* Checks the shared-memory exchange tables the sweep kernel would get for the plan
 * of ops (dtype SC_C64 or SC_C128): each exchange between two stages writes and reads
 * every slot once and agrees on where each amplitude lies.  stats[4] = {exchanges,
 * exchanges with their own swizzle, 128-byte wavefronts, wavefronts with a bank
 * conflict}.  Returns the number of sweeps, or SC_ESTATE if a table is inconsistent. */
SC_API int32_t sc_debug_check_exchanges(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                                 int32_t low_qubits, int32_t nr, int32_t dtype, int64_t* stats);
/* Checks the whole-tile tensor copies (TMA boxes) the sweep kernel would use for the
 * plan of ops over `batch` states: for each sweep whose tile is a box of the state
 * tensor, every tile position of a spread of tiles is copied from the amplitude the
 * sweep's tile enumeration assigns to it.  stats[2] = {sweeps with a box form, tiles
 * checked}.  Returns the number of sweeps, or SC_ESTATE on a mismatch. */
SC_API int32_t sc_debug_check_tile_tensors(int32_t n, const sc_op* ops, int64_t n_ops,
                                           int32_t tile_qubits, int32_t low_qubits, int32_t nr,
                                           int32_t dtype, int64_t batch, int64_t* stats);
/* As sc_debug_emulate_sweeps for one trajectory of a batch: Pauli slot j sits after
 * op slot_after[j] (non-decreasing) on qubit slot_qubit[j] and applies paulis[j]
 * (0 = I, 1 = X, 2 = Y, 3 = Z), planned the way sc_trajectories plans slots. */
SC_API int32_t sc_debug_emulate_slots(int32_t n, const sc_op* ops, int64_t n_ops, int32_t tile_qubits,
                               int32_t low_qubits, int32_t nr, double budget,
                               const int64_t* slot_after, const int32_t* slot_qubit,
                               int64_t n_slots, const uint8_t* paulis, double* state);

#ifdef __cplusplus
}
#endif

#endif /* STATECRAFT_B200_H */
