// knnag_forward_noalloc: the forward with its scratch in a fixed device array.
//
// Some callers cannot allocate device memory at the point where they need
// the op: code running inside an allocator-free section of a serving loop,
// plugins whose host framework owns every device allocation and forbids
// cudaMalloc from extensions, or callers that cannot size or keep a
// workspace buffer.  For them this entry point takes only inputs and
// outputs; the scratch knnag_forward needs (status words, flagged-query
// list, packed point records, search tiles) lives in one file-scope
// `__device__` array of kNoallocScratchBytes that every GPU loading this
// library holds until the process exits.
//
// Host code cannot use the array's name as a device address, so on the
// first call on each device (with that device current) the address is
// looked up once with cudaGetSymbolAddress and cached; that first call
// should therefore come before any stream capture.  All calls share the one
// array: the forward clears what must start at zero (status word and flag
// count) at the start of every call, and two calls that overlap on the GPU
// (different streams, or different threads without ordering) race on it.
// Errors latched on the device (a bounded wait that gave up, an internal
// index out of range) land in the array's first word, which
// knnag_noalloc_read_device_status copies back and clears; the next
// forward call clears it too, so it must be read before that call.  The
// cached address assumes the device's primary context lives as long as the
// process (a cudaDeviceReset would leave it stale).
#include <cuda_runtime.h>

#include <mutex>

#include "knn_aniso.h"
#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {

// 8 MiB: the forward's scratch is about 276 bytes per point (records, search
// tiles, spatial-index keys and permutation, tile infos, the tensor-core
// filter's tile operands) plus 19 bytes per query (flag list, query
// permutation, seed positions, search plan): up to ~31k points with few
// queries, or ~15k points with ~230k queries.
constexpr size_t kNoallocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device); nullptr on failure.
void* noalloc_scratch_on_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_ptr[dev] = ptr;
  }
  return g_noalloc_ptr[dev];
}

}  // namespace
}  // namespace knnag

using namespace knnag;

extern "C" int knnag_forward_noalloc(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                                     int B, int Q, int P, int F, int K, int dtype, void* f_out, void* w_out,
                                     void* dists, int64_t* idxs, void* stream) {
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  if (B < 0 || Q < 0 || P < 0 || F < 0) return KNNAG_ERR_ARG;
  if (K < 1 || K > P) return KNNAG_ERR_K;
  if ((int64_t)B * Q * K > 2147483647LL || (int64_t)B * P > 2147483647LL / kRecLen) return KNNAG_ERR_TOO_LARGE;
  if ((int64_t)B * Q == 0) return KNNAG_OK;
  if (!q || !p || !sigma || !R || !w_out || !dists || !idxs) return KNNAG_ERR_ARG;
  if (F > 0 && (!f || !f_out)) return KNNAG_ERR_ARG;
  if (fwd_layout(B, Q, P, K, dtype, true).total > kNoallocScratchBytes) return KNNAG_ERR_SCRATCH_LIMIT;
  void* scratch = noalloc_scratch_on_current_device();
  if (!scratch) return KNNAG_ERR_CUDA;
  return forward_impl(q, p, f, sigma, R, B, Q, P, F, K, dtype, f_out, w_out, dists, idxs, nullptr, scratch,
                      static_cast<cudaStream_t>(stream));
}

extern "C" int knnag_noalloc_read_device_status(void* stream) {
  void* scratch = noalloc_scratch_on_current_device();
  if (!scratch) return KNNAG_ERR_CUDA;
  // the forward's status word is the first word of its layout
  return knnag_read_device_status(scratch, stream);
}
