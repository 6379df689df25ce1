// Internal declarations shared by the C ABI, the fusion planner and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/statecraft_b200.h"

namespace sc {

// ---------------------------------------------------------------------------
// normalised gates (host)
// ---------------------------------------------------------------------------
// Every unitary sc_op is normalised into one of these before planning:
//   PK_DENSE1  2x2 on q0 (optionally controlled by cmask)      m[0..7]
//   PK_DENSE2  4x4 on (q0 = first, q1 = second)                m[0..31]
//   PK_X       controlled pair swap on target q0 (CNOT / MCX)   -
//   PK_SWAP    swap of qubits q0, q1                            -
//   PK_DIAG1   diag(d0, d1) on q0, optionally controlled        m[0..3]
//   PK_DIAG2   diag(d[4]) on (q0 = first, q1 = second)          m[0..7]
//   PK_PAULI   Pauli slot on q0 (batched trajectories): the Pauli (I, X, Y or Z)
//              is chosen per trajectory; q1 = slot index into the choice table
// PK_PROBE (adjoint reverse pass only): q0 = qubit, q1 = Pauli generator (1 = X,
// 2 = Y, 3 = Z), op_index = gradient slot; adds Im <lambda| P |psi> to that slot.
// PK_TMAT (batched trajectories): a 2x2 matrix on q0 chosen per trajectory on the
// device (a drawn Kraus operator over the square root of its weight); q1 = its
// index among the batch's Kraus points.
enum PKind : int32_t {
  PK_DENSE1 = 0, PK_DENSE2, PK_X, PK_SWAP, PK_DIAG1, PK_DIAG2, PK_PAULI, PK_PROBE, PK_TMAT
};

struct PGate {
  int32_t kind;
  int32_t q0, q1;
  uint64_t cmask;
  double m[32];
  int64_t op_index;
};

// FMA-per-amplitude cost model used by the planner.
double gate_cost(const PGate& g);
uint64_t dense_mask(const PGate& g);
uint64_t touch_mask(const PGate& g);

// Converts one validated sc_op into zero or one PGate (MEASURE -> none).
// params/n_params resolve SC_OP_R* angles.  Returns false for unknown kinds.
bool normalise_op(const sc_op& op, const double* params, int64_t n_params, PGate* out,
                  bool* produced);

// ---------------------------------------------------------------------------
// fused tile sweeps (device-visible plan records)
// ---------------------------------------------------------------------------
// A sweep moves every amplitude through a CTA once.  A tile holds the 2^T
// amplitudes whose indices differ only in the tile qubits: the L lowest qubits
// (tile positions 0..L-1) plus h = T - L "high" qubits hq[] (positions L..T-1).
// Inside the tile, a stage gives each thread 2^NR amplitudes that differ in the
// NR tile positions R[0..NR-1] (ascending); every gate of the stage acts on those
// register bits (dense / permutation kinds) or on any bit (diagonal kinds).
// SK_DP: a two-qubit diagonal that depends only on the parity of its two bits
// (diag(d0, d1, d1, d0), e.g. RZZ / exp(-i g ZZ)); pool holds d0, d1.
// SK_CX: controlled X whose target (a) and one control (b) are register bits; any
//        other controls are tile positions outside the registers (lmask) or global.
// SK_DPR: SK_DP whose two bits are register bits a, b.
// SK_G1ALL: uncontrolled 2x2 gates on several distinct register bits (bit mask in a),
//        matrices in the pool in increasing bit order; they commute, so one record.
// SK_D1R: uncontrolled diag(d0, d1) on register bit a.
// SK_X0 / SK_CX0: SK_X / SK_CX without controls on tile positions outside the
//        registers (a fixed register permutation).
// SK_PAULI: Pauli slot on register bit a; b = slot, the Pauli of each trajectory
//        comes from the sweep's choice table (0 = I, 1 = X, 2 = Y, 3 = Z).
// SK_PAULIF: a Pauli slot conjugated through register permutations folded into the
//        stage's exit permutation; pool (u, w, p) for X, Y, Z in turn: the slot
//        applies i^p X^u Z^w over the register bits (u, w bit masks).
// SK_G1ALLQ: SK_G1ALL in rotation form: each 2x2 unitary is s_g * diag(1, e^{i phi})
//        [[1, -t], [t, 1]] diag(1, e^{i lam}).  Pool: t of each of the K gates, then
//        t / (1 + t^2) of each, then the products of their (1 + t^2) e^{i lam}
//        (the real factor makes each rotation two in-place shears) and of their
//        e^{i phi} over every non-empty
//        subset of the gates (2 x (2^K - 1) complex; bit k of the subset index is the
//        k-th gate in increasing register bit).  The scalars s_g are carried in
//        SwSweep::scale and applied to every amplitude at a sweep's store.  b: register
//        bits whose gate is U X in rotation form (|u00| too small for U itself): the
//        record first applies X on those bits.
// SK_XF / SK_CXF: X on register bit a (controlled by register bit b for CXF) whose
//        other controls lie outside the registers (lmask: tile positions, gmask:
//        global qubits), last to touch its bits in a stage that is not the sweep's
//        last: applied to the stage's exit slots instead of the registers.
// SK_PROBE: gradient probe on register bit a, generator Pauli in the code's low two
//        bits (1 = X, 2 = Y, 3 = Z), b = gradient slot (the adjoint reverse sweep).
// SK_DTAB: a diagonal over the stage's register bits as a table of 2^NR complex
//        factors (register j is multiplied by entry j): adjacent register-bit
//        diagonals of a stage merged into one record.
// SK_TMAT: 2x2 matrix on register bit a read per trajectory from the batch's matrix
//        table (b = Kraus point: entry b * batch + trajectory, 8 reals).
// SK_ROTL: real rotations [[cos al, -sin al], [sin al, cos al]] on the register bits of
//        mask a (plans whose global phase is free, PlanParams::phase_free), each as
//        three in-place shears a0 += p a1, a1 += s a0, a0 += p a1 with p = -tan(al/2),
//        s = sin al, |al| <= pi/2.  Pool: (p, s) per gate in increasing register bit.
// SK_D1H: diag(1, d) on register bit a (a 1-qubit diagonal with its global phase
//        dropped, phase-free plans); pool: d (complex).
enum SwKind : int32_t {
  SK_G1 = 0, SK_G2, SK_X, SK_SWAP, SK_D1, SK_D2, SK_DP, SK_CX, SK_DPR, SK_G1ALL, SK_D1R,
  SK_X0, SK_CX0, SK_PAULI, SK_G1ALLQ, SK_XF, SK_CXF, SK_PROBE, SK_PAULIF, SK_DTAB, SK_TMAT,
  SK_ROTL, SK_D1H
};

// Dispatch code of a sweep gate: kind << 4 | a << 2 | b for kinds whose a / b are
// register bits (< 4), kind << 4 | mask for SK_G1ALL, kind << 4 otherwise.  The
// kernel switches on it once.
inline int32_t sw_code(int32_t kind, int32_t a, int32_t b) {
  switch (kind) {
    case SK_G1: case SK_X: case SK_D1R: case SK_X0: case SK_PAULI: case SK_XF: case SK_TMAT:
    case SK_D1H:
      return (kind << 4) | (a << 2);
    case SK_G2: case SK_SWAP: case SK_CX: case SK_DPR: case SK_CX0: case SK_CXF:
      return (kind << 4) | (a << 2) | b;
    case SK_G1ALL: case SK_G1ALLQ: case SK_ROTL:
      return (kind << 4) | (a & 15);  // a = register-bit mask
    default: return kind << 4;
  }
}

constexpr int SW_MAX_HIGH = 24;
constexpr int SW_MAX_NR = 4;

struct SwGate {     // 32 bytes
  int32_t kind;     // SwKind
  int32_t a, b;     // register bits (G1/G2/X/SWAP) or diagonal qubit refs (D1/D2):
                    //   ref >= 0 -> tile position, ref < 0 -> global qubit (-ref - 1)
  int32_t moff;     // offset of the matrix in the sweep pool (reals)
  uint32_t lmask;   // control bits on tile positions
  int32_t code;     // sw_code(kind, a, b)
  uint64_t gmask;   // control bits on global (non-tile) qubits
};

struct SwStage {    // 32 bytes
  int32_t g0, g1;   // gate range
  int8_t R[SW_MAX_NR];
  int32_t nr;       // number of meaningful register positions (== kernel NR)
  // Exit permutation of the registers: permutation gates on register bits (X,
  // CNOT, SWAP) are not executed but folded here; the data of register j leaves
  // the stage as register perm[j] (through the next exchange or the final store).
  int8_t perm[16];
};

// Qubit layout.  The planner keeps a logical -> physical map of the qubits: the
// amplitude of logical basis index x lives at the physical index whose bit
// phys[q] is bit q of x.  Every sweep reads its tile through the layout in force
// and may write it back through a new one (a "relayout"): up to NR of the tile's
// high qubits move onto the contiguous low physical bits for the sweeps that
// follow, the low qubits they displace take their physical bits.  A plan ends
// with the identity layout; when the last sweep cannot restore it, `restore`
// holds in-place bit permutations that do.
struct SwSweep {
  int32_t T, L, h, nr;
  int32_t s0, s1;            // stage range
  int32_t pool0, pool1;      // range of plan.pool holding this sweep's record data
  int64_t tiles;
  int32_t hq[SW_MAX_HIGH];   // physical bit of tile position L + k (input layout)
  int32_t hs[SW_MAX_HIGH];   // the same physical bits, ascending (tile enumeration)
  int8_t outp[32];           // physical bit tile position p is written to (output layout)
  int32_t relayout;          // outp differs from the input map
  // the rotation-form scalar this sweep applies at its store: the product of its own
  // gates' scalars and those carried from earlier sweeps (1 when it carries them on)
  double scale_re, scale_im;
};

// In-place permutation of physical qubit bits: the tile is the 2^nbits
// amplitudes that differ in bits[0..nbits-1] (ascending), and the content of
// physical bit bits[src[k]] moves to physical bit bits[k] (tile element o takes
// the amplitude of tile element sum_k bit_k(o) << src[k]).  The bit set is closed
// under the permutation, so every tile reads and writes the same addresses.
constexpr int SW_PERM_MAX_BITS = 12;
struct SwPerm {
  int32_t nbits;
  int8_t bits[SW_PERM_MAX_BITS];
  int8_t src[SW_PERM_MAX_BITS];
};

struct PlanParams {
  int tile_qubits;   // T (clamped to n)
  int low_qubits;    // L
  int nr;            // register qubits per stage
  double budget;     // FMA per amplitude per sweep; < 0 unlimited
  int max_gates;     // per sweep
  int max_pool = 1 << 30;  // matrix reals per sweep
  bool relayout = true;    // let sweeps move qubits onto the low physical bits
  // 1-qubit unitaries with |u00| >= rot_min_c use the rotation form (0: never);
  // the bound keeps t = |u10| / |u00| in range
  double rot_min_c = 0.0;
  // smallest magnitude of the rotation-form scalar, both the part a sweep collects
  // and the part carried from earlier sweeps: the stored amplitudes are the true
  // ones divided by the scalar, so they stay below 1 / scale_floor^2
  double scale_floor = 0x1p-200;
  // per-stage record peephole (diagonals merged or moved, permutations folded)
  bool peephole = true;
  // fold the register permutations that open a stage into its read (StageEntry)
  bool entry_fold = true;
  // a common phase of the whole state may be dropped: the adjoint reverse pass
  // applies every gate to both of its states, so a phase e^{ig} (or a sign) on a
  // gate cancels in every probe Im <lambda| P |psi>.  1-qubit real rotations up to
  // a phase become SK_ROTL records and 1-qubit diagonals on register bits SK_D1H.
  bool phase_free = false;
};

// matrix reals a normalised gate stores in the sweep pool
int gate_pool_size(const PGate& g);

// Entry folds of a stage (host side): the register permutations that open a stage
// (X, CNOT and SWAP on register bits, and X on a register bit controlled from outside
// the registers) are not executed as records but folded into the stage's read: the
// thread's register j reads the amplitude of register rperm[j] of the plain read,
// with register-index flip rf_d[k] where the condition of record rf_g[k] holds (its
// global controls gmask on the tile, its tile-position controls lmask on the thread).
// The folded records stay in `gates` just before the stage's range (g_start .. g0).
constexpr int kEntryMaxCond = 2;
struct StageEntry {
  int32_t g_start = 0;  // the stage's first record before folding
  int8_t rperm[16];
  int32_t n_rf = 0;
  int32_t rf_g[kEntryMaxCond] = {-1, -1};
  int32_t rf_d[kEntryMaxCond] = {0, 0};
  StageEntry() {
    for (int j = 0; j < 16; ++j) rperm[j] = (int8_t)j;
  }
};

struct Plan {
  std::vector<SwSweep> sweeps;
  std::vector<SwStage> stages;
  std::vector<StageEntry> entry;  // per stage (empty: no entry folds)
  std::vector<SwGate> gates;
  std::vector<double> pool;
  std::vector<int64_t> gate_ops;  // host only: op index of each entry of `gates`
  std::vector<SwPerm> restore;    // bit permutations back to the identity layout
  int64_t n_gates = 0;
  bool ok = true;  // false if some gate could not be staged (planner invariant broken)
};

// Builds the sweep plan for a gate list on n qubits.
Plan plan_sweeps(const std::vector<PGate>& gates, int n, const PlanParams& pp);

// First record of a sweep, the records its first stage folded into its read included.
inline int32_t sweep_first_gate(const Plan& plan, const SwSweep& sw) {
  return plan.entry.empty() ? plan.stages[sw.s0].g0 : plan.entry[sw.s0].g_start;
}


// ---------------------------------------------------------------------------
// kernel classes (timing / statistics)
// ---------------------------------------------------------------------------
enum KernelClass : int32_t {
  KC_SWEEP = 0,
  KC_GATE_DENSE,
  KC_GATE_PERM,
  KC_GATE_DIAG,
  KC_INIT,
  KC_PROB,
  KC_SAMPLE,
  KC_NOISE,
  KC_EXPECT,
  KC_ADJOINT,
  KC_BATCH,
  KC_PERMUTE,
  KC_BLOCK,
  KC_COUNT
};
const char* kernel_class_name(int cls);

// ---------------------------------------------------------------------------
// launchers (implemented in the .cu files; all asynchronous on `stream`)
// ---------------------------------------------------------------------------
// per-gate path (fusion off); `state` is double2* or float2* per dtype
cudaError_t launch_gate(int dtype, void* state, int n, const PGate& g, cudaStream_t s);
// fused sweep number k of `plan` (n <= 32); `err` (device int) is set to 1 if a
// bulk-copy wait times out
cudaError_t launch_sweep(int dtype, void* state, const Plan& plan, size_t k, int* err,
                         int sm_count, cudaStream_t s);
// the same sweep over `batch` states of n qubits stored back to back; Pauli slots
// read trajectory b's choice of slot j at paulis[b * n_slots + j]; SK_TMAT records
// read their matrix at tmats + (point * batch + b) * 8 (float or double per dtype)
cudaError_t launch_sweep_batch(int dtype, void* states, int n, int64_t batch, const Plan& plan,
                               size_t k, const uint8_t* paulis, int n_slots, const void* tmats,
                               int* err, int sm_count, cudaStream_t s);
// Fused adjoint reverse pass (plans of inverse gates with SK_PROBE records):
// adjoint_plan_supported says whether every sweep fits the dual-state kernel
// (register qubits 3, at least 32 threads per tile, matrix / permutation /
// diagonal records only, no rotation scalar, no layout change); the launcher runs
// sweep k on psi and lambda and adds its probe sums to grad[slot] through
// `partial` (room for max_ctas x kSweepMaxGates doubles).
bool adjoint_plan_supported(const Plan& plan);
// Host check of a plan's shared-memory exchange tables (the layouts the sweep kernel
// uses): every exchange writes and reads each slot once, the slot a writer uses for
// a tile index is the one the reader takes it from, and stats[] = {exchanges,
// exchanges with a non-default swizzle, wavefronts, wavefronts with a bank
// conflict}.  False when the tables are inconsistent or a sweep has no kernel form.
bool check_exchange_tables(const Plan& plan, int dtype, int64_t* stats);
// Host check of the whole-tile tensor copies of a plan's sweeps over `batch` states:
// for each sweep with a box form, every tile position of a spread of work items is
// copied from the amplitude the sweep's tile enumeration assigns to it.  stats[2] =
// {sweeps with a box form, work items checked}.
bool check_tile_tensors(const Plan& plan, int dtype, int64_t batch, int64_t* stats);
cudaError_t launch_adjoint_sweep(int dtype, void* psi, void* lam, const Plan& plan, size_t k,
                                 double* partial, int max_ctas, double* grad, int sm_count,
                                 cudaStream_t s);
// Dense blocks (k_block.cu, sc_blocks.cpp): a run of gates touching k (3..5) qubits
// composed into one 2^k x 2^k complex unitary, applied with FP64 tensor-core tiles.
struct BlockArgs {
  int32_t k;
  int32_t q[5];  // the block's qubits, ascending; local bit b <-> qubit q[b]
};
struct DenseBlock {
  BlockArgs args;
  int32_t n_gates;
  std::vector<double> u;  // 2^k x 2^k row-major, (re, im) pairs
};
// One item of a gate stream cut into sweep-planned runs and dense blocks.
struct GateRun {
  std::vector<PGate> gates;  // planned into sweeps (may be empty)
  int block = -1;            // index into the block list, applied after `gates`
};
// Cuts `gates` into runs and blocks: consecutive gates whose touched qubits fit in
// 5 form a block when their summed gate_cost is at least min_cost (FMA per
// amplitude) and they touch at least 3 qubits; everything else stays in runs.
std::vector<GateRun> cut_dense_blocks(const std::vector<PGate>& gates, int n, double min_cost,
                                      std::vector<DenseBlock>* blocks);
// u: device copy of the block's matrix (2 * 4^k doubles); complex128 states only
cudaError_t launch_block(void* state, int n, const BlockArgs& a, const double* u, int sm_count,
                         cudaStream_t s);
// in-place qubit-bit permutation of an n-qubit state
cudaError_t launch_permute(int dtype, void* state, int n, const SwPerm& perm, int sm_count,
                           cudaStream_t s);
// |0..0> or |basis>
cudaError_t launch_init_basis(int dtype, void* state, int n, uint64_t basis, cudaStream_t s);
// |0..0> in each of `batch` n-qubit states stored back to back
cudaError_t launch_init_batch(int dtype, void* states, int n, int64_t batch, cudaStream_t s);
// c128 host layout -> device amplitudes (dtype conversion for c64)
cudaError_t launch_convert_in(int dtype, void* state, const double* src, int64_t count,
                              cudaStream_t s);
cudaError_t launch_convert_out(int dtype, const void* state, double* dst, int64_t count,
                               cudaStream_t s);

}  // namespace sc
