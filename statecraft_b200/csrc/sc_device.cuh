// Device helpers shared by the kernels: amplitude types, complex arithmetic,
// index bit manipulation and the shared-memory swizzle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sc_rng.h"

namespace sc {

// Amplitude storage: complex128 = double2 (16 B), complex64 = float2 (8 B).
template <typename R> struct Amp;
template <> struct Amp<double> {
  using type = double2;
  // 128-byte shared-memory row = 8 amplitudes
  static constexpr int kSwizzleShift = 3;
};
template <> struct Amp<float> {
  using type = float2;
  static constexpr int kSwizzleShift = 4;
};

template <typename R>
__device__ __forceinline__ typename Amp<R>::type make_amp(R re, R im) {
  typename Amp<R>::type a;
  a.x = re;
  a.y = im;
  return a;
}

// (ar + i ai) * (br + i bi)
template <typename A, typename R>
__device__ __forceinline__ A cmul(R br, R bi, A a) {
  A o;
  o.x = br * a.x - bi * a.y;
  o.y = br * a.y + bi * a.x;
  return o;
}

// m0 * a0 + m1 * a1 with m given as (re, im) pairs
template <typename A, typename R>
__device__ __forceinline__ A cmac2(R m0r, R m0i, A a0, R m1r, R m1i, A a1) {
  A o;
  o.x = m0r * a0.x - m0i * a0.y + m1r * a1.x - m1i * a1.y;
  o.y = m0r * a0.y + m0i * a0.x + m1r * a1.y + m1i * a1.x;
  return o;
}

__host__ __device__ __forceinline__ uint64_t insert_zero64(uint64_t x, int bit) {
  const uint64_t low = x & ((1ULL << bit) - 1ULL);
  return ((x >> bit) << (bit + 1)) | low;
}

__host__ __device__ __forceinline__ uint32_t insert_zero32(uint32_t x, int bit) {
  const uint32_t low = x & ((1u << bit) - 1u);
  return ((x >> bit) << (bit + 1)) | low;
}

// XOR swizzle of shared-memory slots: the 16-byte chunk index inside each
// 128-byte row is XORed with the row index (mod chunks per row).  Stage gathers
// whose lanes stride by whole rows then hit distinct banks.
template <typename R>
__device__ __forceinline__ uint32_t swz(uint32_t i) {
  constexpr int s = Amp<R>::kSwizzleShift;
  return i ^ ((i >> s) & ((1u << s) - 1u));
}

// ---------------------------------------------------------------------------
// Bulk asynchronous copies (TMA, cp.async.bulk) and mbarriers, sm_90+.
// No cluster multicast is used anywhere.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the mbarrier phase with the given parity; gives up after `limit`
// clock cycles and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  long long limit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// global -> shared bulk copy completing on an mbarrier (bytes % 16 == 0, 16-byte aligned)
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Tiled bulk tensor copy (TMA) of one box, global -> shared, completing on an
// mbarrier.  tmap: generic address of a CUtensorMap in kernel-parameter or global
// memory; c[0..rank-1]: box coordinates (innermost first; c[0] must keep the copy
// 16-byte aligned).  No cluster multicast.
__device__ __forceinline__ void tensor_load(void* dst_smem, const void* tmap, const int32_t* c,
                                            int rank, uint64_t* bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(tmap);
  const uint32_t d = smem_u32(dst_smem), b = smem_u32(bar);
  switch (rank) {
    case 1:
      asm volatile(
          "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2}], [%3];" ::"r"(d), "l"(m), "r"(c[0]), "r"(b)
          : "memory");
      break;
    case 2:
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3}], [%4];" ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(b)
          : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]),
          "r"(b)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]),
          "r"(c[2]), "r"(c[3]), "r"(b)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]),
          "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b)
          : "memory");
      break;
  }
}

// Tiled bulk tensor copy of one box, shared -> global, tracked by the issuing
// thread's bulk groups.
__device__ __forceinline__ void tensor_store(const void* tmap, const int32_t* c, int rank,
                                             const void* src_smem) {
  const uint64_t m = reinterpret_cast<uint64_t>(tmap);
  const uint32_t s = smem_u32(src_smem);
  switch (rank) {
    case 1:
      asm volatile("cp.async.bulk.tensor.1d.global.shared::cta.tile.bulk_group [%0, {%1}], [%2];"
                   ::"l"(m), "r"(c[0]), "r"(s)
                   : "memory");
      break;
    case 2:
      asm volatile(
          "cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];"
          ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(s)
          : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];"
          ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(s)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}],"
          " [%5];" ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(s)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4,"
          " %5}], [%6];" ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]),
          "r"(s)
          : "memory");
      break;
  }
}

// shared -> global bulk copy tracked by the issuing thread's bulk groups
__device__ __forceinline__ void bulk_store(void* dst, const void* src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src_smem)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the shared-memory sources of this thread's committed bulk stores have been read
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// this thread's committed bulk stores are complete
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// orders this thread's generic-proxy shared-memory accesses with async-proxy (TMA) ones
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// per-thread asynchronous global -> shared copies (16 or 8 bytes), tracked in
// this thread's cp.async groups
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst_smem, const void* src) {
  static_assert(BYTES == 16 || BYTES == 8, "cp.async size");
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst_smem)), "l"(src)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst_smem)), "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// all but the newest `N` of this thread's cp.async groups have completed
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace sc
