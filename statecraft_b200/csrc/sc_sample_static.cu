// Sampling that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they sample.  A
// framework whose device memory is owned by its own pool allocator cannot let a
// library take memory behind the pool's back; a serving loop that must not stall or
// fail on an allocation after start-up cannot afford one per request; a process
// that has handed almost all of the GPU's memory to its own buffers has nothing
// left for a library to allocate.  They hold the state vector in their own device
// memory and want outcomes written into their own device buffer.
//
// sc_sample_static samples every qubit of such a state (outcome = basis index, the
// countsAll convention) with the same kernels as sc_sample.  Its only scratch -- the
// per-chunk sums, approximate and exact running sums and records of the running sum,
// and the scalars -- lives in the file-scope array below: room for states of up to
// kStaticMaxAmps = 2^30 amplitudes (30 qubits), about 24 MiB that every GPU which
// loads this library holds until the process exits.  Larger states are rejected with
// SC_EINVAL.
//
// The array's name is a host-side stand-in in host code, so its device address is
// looked up with cudaGetSymbolAddress once per device, with that device current,
// on the first call made on it; make that first call before any stream capture.
// The address is kept for the life of the process, so a cudaDeviceReset between
// calls is not supported (the reset frees the module that holds the array).
// Every call shares the array and it keeps the previous call's contents; the
// kernels write every word they read earlier in the same call, so nothing needs
// clearing, but calls that overlap on the GPU race on the array.  Each call waits
// for its stream and reads a status word back before it returns, so a call on a
// stream that is capturing returns SC_EINVAL before it enqueues anything.
#include <cuda_runtime.h>

#include <mutex>

#include "sc_ctx.h"
#include "sc_measure.h"

namespace sc {

namespace {

constexpr uint64_t kStaticMaxAmps = 1ULL << 30;
constexpr uint64_t kStaticChunks = kStaticMaxAmps / kSampleChunk;
// layout: chunk sums | approximate running sums | exact running sums [kStaticChunks
// doubles each] | chunk records [kStaticChunks ChunkTf] | scalars
static_assert(sizeof(ChunkTf) % sizeof(double) == 0, "records pack into doubles");
constexpr uint64_t kTfDoubles = sizeof(ChunkTf) / sizeof(double);
constexpr uint64_t kStaticDoubles = (3 + kTfDoubles) * kStaticChunks + 8;
static_assert(sizeof(SampleScalars) <= 8 * sizeof(double), "scalars must fit the tail");

static __device__ __align__(256) double g_sample_scratch[kStaticDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

int scratch_for(int device, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_sample_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(sample scratch)");
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return SC_OK;
}

}  // namespace

}  // namespace sc

using namespace sc;

extern "C" int32_t sc_sample_static(const void* d_state, int32_t n_qubits, int32_t dtype,
                                    int64_t shots, uint64_t seed, const double* d_uniforms,
                                    int32_t* d_outcomes, void* stream) {
  if (!d_state || !d_outcomes) return fail(SC_EINVAL, "state and outcome buffers are required");
  if (dtype != SC_C128 && dtype != SC_C64) return fail(SC_EINVAL, "dtype must be SC_C128 or SC_C64");
  if (n_qubits < 1) return fail(SC_EINVAL, "qubitCount must be positive");
  // the qubit count is bounded before it is used as a shift
  if (n_qubits > 30 || (1ULL << n_qubits) > kStaticMaxAmps)
    return fail(SC_EINVAL, "sc_sample_static supports states of up to 2^30 amplitudes (30 qubits), got %d qubits",
                n_qubits);
  if (shots <= 0) return fail(SC_EINVAL, "shots must be positive");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the call ends by waiting for the stream, which a capturing stream does not
  // allow (and the wait would invalidate the caller's capture): refuse before any
  // work is enqueued or the scratch array is looked up
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return fail_cuda(e, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fail(SC_EINVAL, "sc_sample_static waits for its stream and cannot be called while the stream is capturing");
  int device = 0;
  e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) return fail(SC_EINVAL, "device ordinal %d out of range", device);
  double* scratch = nullptr;
  int rc = scratch_for(device, &scratch);
  if (rc != SC_OK) return rc;
  int sms = 148;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
    return fail_cuda(e, "cudaDeviceGetAttribute");
  SampleArgs a;
  a.chunk_sums = scratch;
  a.chunk_prefix = scratch + kStaticChunks;
  a.chunk_start = scratch + 2 * kStaticChunks;
  a.chunk_tf = reinterpret_cast<ChunkTf*>(scratch + 3 * kStaticChunks);
  a.scalars = reinterpret_cast<SampleScalars*>(scratch + (3 + kTfDoubles) * kStaticChunks);
  a.uniforms = d_uniforms;
  a.seed = seed;
  a.shots = shots;
  a.outcomes = d_outcomes;
  a.sm_count = sms;
  if ((e = launch_sample(dtype, d_state, nullptr, 1ULL << n_qubits, a, s)) != cudaSuccess)
    return fail_cuda(e, "sampling kernels");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail_cuda(e, "sc_sample_static");
  SampleScalars host;
  if ((e = cudaMemcpy(&host, a.scalars, sizeof host, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "sampler status");
  if (host.status != 0) return fail(SC_ESTATE, "State collapsed to zero probability amplitudes");
  return SC_OK;
}
