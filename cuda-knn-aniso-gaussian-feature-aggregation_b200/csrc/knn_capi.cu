// C ABI of libknn_aniso.so (declared in include/knn_aniso.h): argument
// validation, workspace sizing, and dispatch to the kernels.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "knn_aniso.h"
#include "knn_common.cuh"
#include "knn_internal.h"

using namespace knnag;

namespace knnag {

static std::atomic<long long> g_launches{0};
static std::atomic<void*> g_ev_begin{nullptr}, g_ev_end{nullptr};

void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static std::atomic<int> g_search_splits{0};
int search_splits_setting() { return g_search_splits.load(std::memory_order_relaxed); }

static std::atomic<int> g_stall_visit{-1}, g_wait_spins{kWaitSpinsDefault};
void apply_search_debug(SearchParams& sp) {
  sp.stall_visit = g_stall_visit.load(std::memory_order_relaxed);
  sp.wait_spins = g_wait_spins.load(std::memory_order_relaxed);
}

// Record a profiling event on `st`: as an external event node while the
// stream is being captured into a graph, as a plain record otherwise.  A
// failed record is cleared so it cannot be mistaken for a launch error.
static void record_profile_event(void* e, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const cudaError_t rc = (cs == cudaStreamCaptureStatusActive)
                             ? cudaEventRecordWithFlags(static_cast<cudaEvent_t>(e), st, cudaEventRecordExternal)
                             : cudaEventRecord(static_cast<cudaEvent_t>(e), st);
  if (rc != cudaSuccess) cudaGetLastError();
}

void profile_begin(cudaStream_t st) {
  void* e = g_ev_begin.load();
  if (e && g_ev_end.load()) record_profile_event(e, st);
}

void profile_end(cudaStream_t st) {
  void* e = g_ev_end.load();
  if (e && g_ev_begin.load()) record_profile_event(e, st);
}

}  // namespace knnag

namespace {

// 16 independent FMA chains per thread: FP32-pipe bound.
__global__ void fp32_peak_kernel(float* out, int iters) {
  float v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = threadIdx.x * 1e-3f + i;
  const float a = 0.999f, b = 1e-4f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __fmaf_rn(v[i], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) s += v[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

constexpr int64_t kI32Max = 2147483647;

int check_sizes(int B, int Q, int P, int F, int K) {
  if (B < 0 || Q < 0 || P < 0 || F < 0) return KNNAG_ERR_ARG;
  if (K < 1 || K > P) return KNNAG_ERR_K;
  if ((int64_t)B * Q * K > kI32Max || (int64_t)B * P > kI32Max / kRecLen ||
      (int64_t)B * round_up(P, kTilePoints) * kRecLen > kI32Max * 4LL)
    return KNNAG_ERR_TOO_LARGE;
  return KNNAG_OK;
}

inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

extern "C" {

const char* knnag_status_string(int status) {
  switch (status) {
    case KNNAG_OK: return "ok";
    case KNNAG_ERR_ARG: return "invalid argument (null pointer or negative size)";
    case KNNAG_ERR_K: return "K must satisfy 1 <= K <= P";
    case KNNAG_ERR_DTYPE: return "unsupported dtype (float32 or float64 only)";
    case KNNAG_ERR_WORKSPACE: return "workspace too small or not 16-byte aligned";
    case KNNAG_ERR_TOO_LARGE: return "problem exceeds the 32-bit entry index range";
    case KNNAG_ERR_CUDA: return "CUDA launch failed";
    case KNNAG_ERR_DEVICE:
      return "device-side error latched (a bounded wait gave up, or a segment table failed validation)";
    case KNNAG_ERR_SCRATCH_LIMIT: return "problem needs more scratch than knnag_forward_noalloc's fixed 8 MiB array";
    default: return "unknown status";
  }
}

int knnag_version(void) { return 10000; }

size_t knnag_forward_workspace_bytes(int B, int Q, int P, int F, int K, int dtype) {
  (void)F;
  if (B < 0 || Q < 0 || P < 0 || K < 1) return 0;
  return fwd_layout(B, Q, P, K, dtype, true).total;
}

size_t knnag_points_bytes(int B, int P, int dtype) {
  return (size_t)B * P * kRecLen * (dtype == KNNAG_F64 ? 8 : 4);
}

size_t knnag_adjacency_bytes(int B, int Q, int P, int K) { return adj_layout(B, Q, P, K).total; }

size_t knnag_backward_workspace_bytes(int B, int Q, int P, int F, int K, int dtype) {
  return bwd_layout(B, Q, P, F, K, dtype).total;
}

int knnag_forward(const void* q, const void* p, const void* f, const void* sigma, const void* R, int B, int Q,
                  int P, int F, int K, int dtype, void* f_out, void* w_out, void* dists, int64_t* idxs,
                  void* points, void* workspace, size_t workspace_bytes, void* stream) {
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  int rc = check_sizes(B, Q, P, F, K);
  if (rc) return rc;
  if ((int64_t)B * Q == 0) return KNNAG_OK;
  if (!q || !p || !sigma || !R || !w_out || !dists || !idxs || !workspace) return KNNAG_ERR_ARG;
  if (F > 0 && (!f || !f_out)) return KNNAG_ERR_ARG;
  if (workspace_bytes < fwd_layout(B, Q, P, K, dtype, points == nullptr).total || !aligned16(workspace) ||
      (points && !aligned16(points)))
    return KNNAG_ERR_WORKSPACE;
  return forward_impl(q, p, f, sigma, R, B, Q, P, F, K, dtype, f_out, w_out, dists, idxs, points, workspace,
                      static_cast<cudaStream_t>(stream));
}

int knnag_forward_counted(const void* q, const void* p, const void* f, const void* sigma, const void* R, int B,
                          int Q, int P, int F, int K, int dtype, void* f_out, void* w_out, void* dists, int64_t* idxs,
                          void* points, void* adjacency, void* workspace, size_t workspace_bytes, void* stream) {
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  int rc = check_sizes(B, Q, P, F, K);
  if (rc) return rc;
  if ((int64_t)B * Q == 0) return KNNAG_OK;
  if (!q || !p || !sigma || !R || !w_out || !dists || !idxs || !workspace || !adjacency) return KNNAG_ERR_ARG;
  if (F > 0 && (!f || !f_out)) return KNNAG_ERR_ARG;
  if (workspace_bytes < fwd_layout(B, Q, P, K, dtype, points == nullptr).total || !aligned16(workspace) ||
      (points && !aligned16(points)) || !aligned16(adjacency))
    return KNNAG_ERR_WORKSPACE;
  return forward_impl(q, p, f, sigma, R, B, Q, P, F, K, dtype, f_out, w_out, dists, idxs, points, workspace,
                      static_cast<cudaStream_t>(stream), adjacency);
}

int knnag_build_adjacency_counted(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, void* stream) {
  int rc = check_sizes(B, Q, P, 0, K);
  if (rc) return rc;
  if (!adjacency || (!idxs && (int64_t)B * Q > 0)) return KNNAG_ERR_ARG;
  if ((int64_t)B * P == 0) return KNNAG_OK;
  return launch_build_adjacency(idxs, B, Q, P, K, adjacency, static_cast<cudaStream_t>(stream), true);
}

int knnag_pack_points(const void* p, const void* sigma, const void* R, int B, int P, int dtype, void* points,
                      void* stream) {
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  if (B < 0 || P < 0) return KNNAG_ERR_ARG;
  if ((int64_t)B * P == 0) return KNNAG_OK;
  if (!p || !sigma || !R || !points || !aligned16(points)) return KNNAG_ERR_ARG;
  return launch_pack_points(p, sigma, R, B, P, dtype, points, static_cast<cudaStream_t>(stream));
}

int knnag_build_adjacency(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, void* stream) {
  int rc = check_sizes(B, Q, P, 0, K);
  if (rc) return rc;
  if (!adjacency || (!idxs && (int64_t)B * Q > 0)) return KNNAG_ERR_ARG;
  if ((int64_t)B * P == 0) return KNNAG_OK;
  return launch_build_adjacency(idxs, B, Q, P, K, adjacency, static_cast<cudaStream_t>(stream));
}

static int backward_common(BwdArgs& x, size_t workspace_bytes, void* stream) {
  if (x.dtype != KNNAG_F32 && x.dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  int rc = check_sizes(x.B, x.Q, x.P, x.F, x.K);
  if (rc) return rc;
  if (x.needs & ~(KNNAG_NEED_ALL | KNNAG_GFO_SCALAR)) return KNNAG_ERR_ARG;
  if ((int64_t)x.B * x.Q == 0 && (int64_t)x.B * x.P == 0) return KNNAG_OK;
  if (!x.gfo || !x.q || !x.p || !x.sigma || !x.R || !x.idxs || !x.workspace) return KNNAG_ERR_ARG;
  if (x.F > 0 && !x.f) return KNNAG_ERR_ARG;
  if (x.order == 2 && !x.ggq) return KNNAG_ERR_ARG;
  if (x.points && !aligned16(x.points)) return KNNAG_ERR_ARG;  // records are read with 16-byte loads
  if (((x.needs & KNNAG_NEED_DQ) && !x.dq) || ((x.needs & KNNAG_NEED_DP) && !x.dp) ||
      ((x.needs & KNNAG_NEED_DF) && !x.df && x.F > 0) || ((x.needs & KNNAG_NEED_DSIGMA) && !x.dsigma) ||
      ((x.needs & KNNAG_NEED_DR) && !x.dR) || ((x.needs & KNNAG_NEED_DGFO) && !x.dgfo && x.F > 0))
    return KNNAG_ERR_ARG;
  if (workspace_bytes < bwd_layout(x.B, x.Q, x.P, x.F, x.K, x.dtype).total || !aligned16(x.workspace))
    return KNNAG_ERR_WORKSPACE;
  return backward_impl(x, static_cast<cudaStream_t>(stream));
}

int knnag_backward(const void* grad_f_out, const void* grad_w_out, const void* q, const void* p, const void* f,
                   const void* sigma, const void* R, const void* w_out, const int64_t* idxs, int B, int Q, int P,
                   int F, int K, int dtype, int needs, const void* points, const void* adjacency, void* dq,
                   void* dp, void* df, void* dsigma, void* dR, void* coef_out, void* workspace,
                   size_t workspace_bytes, void* stream) {
  (void)grad_w_out;  // ignored, as in the reference
  BwdArgs x{};
  x.order = 1;
  x.gfo = grad_f_out;
  x.q = q;
  x.p = p;
  x.f = f;
  x.sigma = sigma;
  x.R = R;
  x.w_in = w_out;
  x.idxs = idxs;
  x.B = B;
  x.Q = Q;
  x.P = P;
  x.F = F;
  x.K = K;
  x.dtype = dtype;
  x.needs = needs & ~KNNAG_NEED_DGFO;
  x.points = points;
  x.adjacency = adjacency;
  x.dq = dq;
  x.dp = dp;
  x.df = df;
  x.dsigma = dsigma;
  x.dR = dR;
  x.coef_out = coef_out;
  x.workspace = workspace;
  return backward_common(x, workspace_bytes, stream);
}

int knnag_backward_2nd(const void* grad_grad_q, const void* grad_f_out, const void* grad_w_out, const void* q,
                       const void* p, const void* f, const void* sigma, const void* R, const void* w_out,
                       const int64_t* idxs, int B, int Q, int P, int F, int K, int dtype, int needs,
                       const void* points, const void* adjacency, const void* coef, void* dgfo, void* dq, void* dp,
                       void* df, void* dsigma, void* dR, void* workspace, size_t workspace_bytes, void* stream) {
  (void)grad_w_out;
  BwdArgs x{};
  x.order = 2;
  x.ggq = grad_grad_q;
  x.gfo = grad_f_out;
  x.q = q;
  x.p = p;
  x.f = f;
  x.sigma = sigma;
  x.R = R;
  x.w_in = w_out;
  x.idxs = idxs;
  x.B = B;
  x.Q = Q;
  x.P = P;
  x.F = F;
  x.K = K;
  x.dtype = dtype;
  x.needs = needs;
  x.points = points;
  x.adjacency = adjacency;
  x.coef_in = coef;
  x.dgfo = dgfo;
  x.dq = dq;
  x.dp = dp;
  x.df = df;
  x.dsigma = dsigma;
  x.dR = dR;
  x.workspace = workspace;
  return backward_common(x, workspace_bytes, stream);
}

size_t knnag_variant_workspace_bytes(int B, int Q, int P, int dtype) {
  if (B < 0 || Q < 0 || P < 0) return 0;
  return 256 + align256((size_t)B * P * kRecLen * (dtype == KNNAG_F64 ? 8 : 4)) + align256((size_t)B * Q * 4);
}

static int variant_checks(const void* q, const void* p, const void* f, const void* sigma, int B, int Q, int P, int F,
                          int K, int dtype, const void* f_out, const void* w_out, const void* dists) {
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  int rc = check_sizes(B, Q, P, F, K);
  if (rc) return rc;
  if ((int64_t)B * Q == 0) return -1;  // nothing to do
  if (!q || !p || !sigma || !w_out || !dists) return KNNAG_ERR_ARG;
  if (F > 0 && (!f || !f_out)) return KNNAG_ERR_ARG;
  return KNNAG_OK;
}

int knnag_forward_precomputed(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                              const int64_t* knn_idxs, int B, int Q, int P, int F, int K, int dtype, void* f_out,
                              void* w_out, void* dists, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = variant_checks(q, p, f, sigma, B, Q, P, F, K, dtype, f_out, w_out, dists);
  if (rc) return rc < 0 ? KNNAG_OK : rc;
  if (!R || !knn_idxs || !workspace) return KNNAG_ERR_ARG;
  if (workspace_bytes < knnag_variant_workspace_bytes(B, Q, P, dtype) || ((uintptr_t)workspace & 15u))
    return KNNAG_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  void* rec = static_cast<char*>(workspace) + 256;
  rc = launch_pack_points(p, sigma, R, B, P, dtype, rec, st);
  if (rc) return rc;
  return variants_precomputed(q, f, rec, knn_idxs, B, Q, P, F, K, dtype, f_out, w_out, dists, st);
}

int knnag_forward_lookup(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                         const int64_t* knn_table, int table_cols, int B, int Q, int P, int F, int K, int dtype,
                         void* f_out, void* w_out, void* dists, int64_t* idxs, void* workspace,
                         size_t workspace_bytes, void* stream) {
  int rc = variant_checks(q, p, f, sigma, B, Q, P, F, K, dtype, f_out, w_out, dists);
  if (rc) return rc < 0 ? KNNAG_OK : rc;
  if (!R || !knn_table || !idxs || !workspace || table_cols < K) return KNNAG_ERR_ARG;
  if (workspace_bytes < knnag_variant_workspace_bytes(B, Q, P, dtype) || ((uintptr_t)workspace & 15u))
    return KNNAG_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  void* rec = ws + 256;
  int* nearest = reinterpret_cast<int*>(ws + 256 + align256((size_t)B * P * kRecLen * (dtype == KNNAG_F64 ? 8 : 4)));
  rc = launch_pack_points(p, sigma, R, B, P, dtype, rec, st);
  if (rc) return rc;
  return variants_lookup(q, p, f, rec, knn_table, table_cols, B, Q, P, F, K, dtype, nearest, f_out, w_out, dists, idxs, st);
}

int knnag_forward_isotropic(const void* q, const void* p, const void* f, const void* sigma, int sigma_cols, int B,
                            int Q, int P, int F, int K, int dtype, void* f_out, void* w_sum, void* dists,
                            int64_t* idxs, void* stream) {
  int rc = variant_checks(q, p, f, sigma, B, Q, P, F, K, dtype, f_out, w_sum, dists);
  if (rc) return rc < 0 ? KNNAG_OK : rc;
  if (!idxs || sigma_cols < 1) return KNNAG_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == KNNAG_F64) {
    ExactParams<double> e{(const double*)q, nullptr, (const double*)f, (const double*)p, (const double*)sigma,
                          sigma_cols, B, Q, P, F, K, 0, nullptr, nullptr, (double*)f_out, (double*)w_sum,
                          (double*)dists, idxs};
    return launch_exact<double>(e, st);
  }
  ExactParams<float> e{(const float*)q, nullptr, (const float*)f, (const float*)p, (const float*)sigma, sigma_cols,
                       B, Q, P, F, K, 0, nullptr, nullptr, (float*)f_out, (float*)w_sum, (float*)dists, idxs};
  return launch_exact<float>(e, st);
}

int knnag_read_device_status(void* workspace, void* stream) {
  if (!workspace) return KNNAG_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int h = 0;
  if (cudaMemcpyAsync(&h, workspace, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return KNNAG_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return KNNAG_ERR_CUDA;
  if (h != 0) {
    cudaMemsetAsync(workspace, 0, sizeof(int), st);
    return KNNAG_ERR_DEVICE;
  }
  return KNNAG_OK;
}

void knnag_set_profile_events(void* ev_begin, void* ev_end) {
  g_ev_begin.store(ev_begin);
  g_ev_end.store(ev_end);
}

long long knnag_launch_count(void) { return g_launches.load(); }

int knnag_set_search_splits(int splits) {
  if (splits != 0 && !search_setting_ok(splits)) return KNNAG_ERR_ARG;
  g_search_splits.store(splits, std::memory_order_relaxed);
  return KNNAG_OK;
}

int knnag_get_search_splits(void) { return g_search_splits.load(std::memory_order_relaxed); }

int knnag_debug_set_search_stall(int visit, int wait_spins) {
  if (visit < -1 || wait_spins < 0) return KNNAG_ERR_ARG;
  g_stall_visit.store(visit, std::memory_order_relaxed);
  g_wait_spins.store(wait_spins > 0 ? wait_spins : kWaitSpinsDefault, std::memory_order_relaxed);
  return KNNAG_OK;
}

int knnag_fp32_peak_probe(float* out, int blocks, int iters, void* stream) {
  if (!out || blocks < 1 || iters < 1) return KNNAG_ERR_ARG;
  fp32_peak_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, iters);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

}  // extern "C"
