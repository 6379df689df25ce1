// Kernel-parameter form of one fused sweep (k_sweep.cu).
#pragma once

#include <stdint.h>

#include "sc_internal.h"

namespace sc {

// A sweep's plan travels as one __grid_constant__ kernel parameter (< 32 KB).
constexpr int kSweepMaxStages = 80;
constexpr int kSweepMaxGates = 78;   // stages <= gates + 2
constexpr int kSweepMaxPool = 2048;  // matrix reals

// Per-stage register tables computed on the host.  off[j] below is the tile offset
// of register j (the OR of 1 << R[k] over the set bits k of j); rd[j] is the slot
// register j is read from, relative to the stage's read base (the thread's l0 in
// the linear layout for stage 0, its swizzled l0 otherwise): the slot of tile
// offset off[j ^ xm], xm being the leading X of the stage's rotation record when
// that record is the stage's only register record (folded into the read; the
// record then skips it), else 0.  wsoff[j] is the slot register j is written to
// when the stage ends (register perm[j] in the next stage's layout) and xoff[a] the
// offset of register bit a in that layout (slot folds).  Each exchange between two
// stages has its own XOR swizzle, slot(i) = i ^ sum_k parity(i & rows[k]) << k over
// the low K slot bits (K = log2 of the amplitudes per 128-byte row); rows[] only
// read bits >= K, so every swizzle is a bijection and XOR-linear over disjoint bits.
// rows[] here is the swizzle of the layout this stage reads; bit 15 of rows[0]
// marks one that differs from the fixed default (rows[k] = 1 << (K + k)).
// Entry folds (StageEntry in the plan) are already in rd[]; their conditional part:
// where the condition of record rf_g[k] (its gmask on the tile, its lmask on the
// thread) holds, the thread's read slots are XORed with rf_off[k] (rf_g[k] < 0: none).
struct SwStageTab {
  uint16_t rd[16];
  uint16_t wsoff[16];
  uint16_t xoff[4];
  uint16_t rows[4];
  int8_t xm;
  int8_t rf_g[2];
  int8_t pad;
  uint16_t rf_off[2];
};

// Whole-tile bulk tensor copies (TMA).  The state is described to the copy engine
// as a tensor of at most kTileTensorMaxRank dims, one per run of consecutive
// physical bits that are all tile bits (copied whole: box = the run) or all
// non-tile bits (box 1), plus one for the state index of a batch.  A tile is then
// one box, landing in shared memory in the order of its physical bits, which is the
// linear tile layout when the high tile qubits are in ascending physical order.
// Coordinate k of work item `it` (state << tiles_log2 | tile) is
// (it >> tm_shift[k]) & tm_mask[k]; tile dims have mask 0.
constexpr int kTileTensorMaxRank = 5;

template <typename R>
struct SweepParams {
  alignas(64) uint64_t tmap[16];  // CUtensorMap (opaque, 128 bytes) when tm_rank > 0
  int32_t tm_rank;
  // failure-detection test hook: when > 0, each CTA's first tile wait is on a barrier
  // nothing arrives on, bounded by this many cycles (the wait runs out)
  int32_t stall_first;
  int32_t tm_shift[kTileTensorMaxRank];
  uint32_t tm_mask[kTileTensorMaxRank];
  int32_t T, L, h, nr;
  int32_t n_stages, relayout;
  int64_t tiles;
  // batched trajectories: `batch` states of 2^nq amplitudes back to back; Pauli
  // slot j of state b applies paulis[b * n_slots + j]
  int32_t nq, n_slots;
  int32_t tiles_log2, pad2;
  int64_t batch;
  const uint8_t* paulis;
  const R* tmats;  // per-trajectory matrices of SK_TMAT records (point * batch + state)
  int32_t pool_len;                      // matrix reals of this sweep (staged in shared memory)
  int32_t n_local_slots;                 // Pauli slots in this sweep
  int32_t slot_map[kSweepMaxGates + 1];  // local slot -> slot index of the choice table
  int32_t hq[SW_MAX_HIGH];  // physical bit of tile position L + k (input layout)
  int32_t hs[SW_MAX_HIGH];  // the same bits ascending (tile enumeration)
  uint8_t outp[32];         // physical bit of tile position p in the output layout
  uint16_t off0[16];     // tile offset of register j in the first stage (linear layout)
  uint32_t gfirst[16];   // global offset of register j in the first stage's layout
  uint32_t gread0[16];   // global offset register j reads in the first stage (entry folds applied)
  uint32_t rf_goff0[2];  // the first stage's conditional entry flips as global offsets
  uint32_t glast[16];    // global offset register j is stored to (last stage, perm applied)
  uint16_t lastoff[16];  // tile offset register j is stored to (last stage, perm applied)
  R scale_re, scale_im;  // applied to every amplitude at the store (rotation-form scalars)
  int32_t has_scale, pad3;
  SwStage stages[kSweepMaxStages];
  SwStageTab tabs[kSweepMaxStages];
  SwGate gates[kSweepMaxGates];
  R pool[kSweepMaxPool];
};

static_assert(sizeof(SweepParams<double>) < 32000, "sweep parameters must fit the 32 KB limit");

}  // namespace sc
