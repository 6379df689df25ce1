// Dense blocks on the FP64 tensor cores (DMMA).
//
// A run of gates that together touch k <= 5 qubits is one 2^k x 2^k complex unitary
// U (composed on the host).  Applying it is a real contraction: the state splits
// into 2^(n-k) columns of 2^k amplitudes (the indices that differ only in the block's
// qubits), and Y = U X for every column, i.e. Yr = Ur Xr - Ui Xi, Yi = Ur Xi + Ui Xr.
// Each warp takes 8 columns at a time and runs the four real products as
// mma.sync.m8n8k4 FP64 tiles (8 rows of Y x 8 columns per tile, k-steps of 4 rows of
// X): D/8 row tiles x D/4 k-steps x 4 products per 8 columns.  U (real and imaginary
// parts) is staged once per CTA in shared memory; each warp stages its 8 columns in a
// shared slab (coalesced: for one row, the 8 columns are consecutive when the lowest
// qubit is not in the block), keeps its B fragments in registers, and writes Y back
// through the same slab.  Slab rows are padded to 9 entries (the fragment stores of
// 8 rows x 4 lanes hit distinct 16-byte bank groups) and U's rows to D + 4 doubles
// (the A fragments' 4 rows x 4 columns per half-warp hit distinct banks).
// complex128 only (complex64 states keep the sweep path).
#include <algorithm>

#include "sc_device.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

constexpr int kBlockWarps = 8;
constexpr int kSlabRow = 9;  // slab row stride in entries (8 columns + 1 pad)

// D = 2^k rows and columns of U; BlockArgs carries the block's qubits (ascending)
template <int D>
__global__ void __launch_bounds__(kBlockWarps * 32)
    k_block(double2* __restrict__ st, int n, BlockArgs a, const double* __restrict__ u) {
  constexpr int KT = D / 4;   // k-steps
  constexpr int MT = D / 8;   // row tiles
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* const ur = reinterpret_cast<double*>(smem_raw);  // [D][D]
  constexpr int UR = D + 4;  // U row stride in doubles
  double* const ui = ur + D * UR;
  double2* const slabs = reinterpret_cast<double2*>(ui + D * UR);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2* const xs = slabs + warp * (D * kSlabRow);  // [row][col]
  for (int e = threadIdx.x; e < D * D; e += blockDim.x) {
    const int at = (e / D) * UR + e % D;
    ur[at] = u[2 * e];
    ui[at] = u[2 * e + 1];
  }
  __syncthreads();
  const int k = a.k;
  // offset of row j: its bits spread over the block's qubits
  auto row_off = [&](int j) {
    uint64_t o = 0;
    for (int b = 0; b < k; ++b)
      if ((j >> b) & 1) o |= 1ULL << a.q[b];
    return o;
  };
  // base of column c: its bits spread over the other qubits
  auto col_base = [&](uint64_t c) {
    uint64_t x = c;
    for (int b = 0; b < k; ++b) x = insert_zero64(x, a.q[b]);
    return x;
  };
  const uint64_t cols = 1ULL << (n - k);
  const uint64_t groups = cols / 8;
  // lane -> (column ln, rows lr, lr + 4, ...) for the loads and stores of the slab
  const int ln = lane & 7, lr = lane >> 3;
  for (uint64_t gidx = (uint64_t)blockIdx.x * kBlockWarps + warp; gidx < groups;
       gidx += (uint64_t)gridDim.x * kBlockWarps) {
    const uint64_t base = col_base(gidx * 8 + ln);
#pragma unroll
    for (int j = lr; j < D; j += 4) xs[j * kSlabRow + ln] = st[base | row_off(j)];
    __syncwarp();
    // B fragments (4 x 8, column-major): lane holds row kt*4 + lane%4, column lane/4
    double br[KT], bi[KT];
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
      const double2 x = xs[(kt * 4 + (lane & 3)) * kSlabRow + (lane >> 2)];
      br[kt] = x.x;
      bi[kt] = x.y;
    }
    __syncwarp();
#pragma unroll 1
    for (int mt = 0; mt < MT; ++mt) {
      double yr0 = 0.0, yr1 = 0.0, yi0 = 0.0, yi1 = 0.0, zr0 = 0.0, zr1 = 0.0;
#pragma unroll
      for (int kt = 0; kt < KT; ++kt) {
        // A fragment (8 x 4, row-major): lane holds row lane/4, column lane%4
        const int ao = (mt * 8 + (lane >> 2)) * UR + kt * 4 + (lane & 3);
        const double ar = ur[ao], ai = ui[ao];
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(yr0), "+d"(yr1) : "d"(ar), "d"(br[kt]));
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(zr0), "+d"(zr1) : "d"(ai), "d"(bi[kt]));
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(yi0), "+d"(yi1) : "d"(ar), "d"(bi[kt]));
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(yi0), "+d"(yi1) : "d"(ai), "d"(br[kt]));
      }
      // C fragment (8 x 8): lane holds row lane/4, columns 2 (lane%4) and 2 (lane%4) + 1
      const int row = mt * 8 + (lane >> 2), c0 = 2 * (lane & 3);
      xs[row * kSlabRow + c0] = make_double2(yr0 - zr0, yi0);
      xs[row * kSlabRow + c0 + 1] = make_double2(yr1 - zr1, yi1);
    }
    __syncwarp();
#pragma unroll
    for (int j = lr; j < D; j += 4) st[base | row_off(j)] = xs[j * kSlabRow + ln];
    __syncwarp();
  }
}

template <int D>
cudaError_t launch_d(double2* st, int n, const BlockArgs& a, const double* u, int sm_count,
                     cudaStream_t s) {
  const size_t smem =
      2 * sizeof(double) * D * (D + 4) + sizeof(double2) * D * kSlabRow * kBlockWarps;
  auto kern = k_block<D>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlockWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const uint64_t groups = (1ULL << (n - a.k)) / 8;
  const uint64_t want = (groups + kBlockWarps - 1) / kBlockWarps;
  const int64_t grid = std::max<int64_t>(
      1, std::min<int64_t>((int64_t)want, (int64_t)sm_count * std::max(per_sm, 1)));
  kern<<<(unsigned)grid, kBlockWarps * 32, smem, s>>>(st, n, a, u);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_block(void* state, int n, const BlockArgs& a, const double* u, int sm_count,
                         cudaStream_t s) {
  if (a.k < 3 || a.k > 5 || n < a.k + 3) return cudaErrorInvalidValue;
  double2* st = static_cast<double2*>(state);
  switch (a.k) {
    case 3: return launch_d<8>(st, n, a, u, sm_count, s);
    case 4: return launch_d<16>(st, n, a, u, sm_count, s);
    default: return launch_d<32>(st, n, a, u, sm_count, s);
  }
}

}  // namespace sc
