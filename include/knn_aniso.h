/*
 * knn_aniso.h -- C ABI of the B200 (sm_100a) anisotropic-Gaussian kNN feature
 * aggregation library (libknn_aniso.so).
 *
 * Computes, for queries q [B,Q,3] against points p [B,P,3] carrying features
 * f [B,P,F], precisions sigma [B,P,3] and axes R [B,P,3,3] (row-major, rows
 * are the axes):
 *     s(q,i)  = sum_a sigma[i][a] * (R[i][a] . (q - p[i]))^2
 *     idxs    = the K points with the smallest s, ascending (ties broken
 *               exactly as the reference's MinK structure breaks them)
 *     dists   = s at those points;  w_out = exp(-dists)
 *     f_out   = sum_k w_out[k] * f[idxs[k]]   (accumulated in k order)
 * and the first- and second-order (Eikonal, through dL/dq) adjoints.
 *
 * Conventions shared by every entry point:
 *   - all tensor pointers are DEVICE pointers to dense row-major arrays;
 *   - dtype selects float32 (KNNAG_F32) or float64 (KNNAG_F64) for every
 *     floating-point array; idxs are int64;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); every launch
 *     goes to it, nothing synchronises the host, nothing allocates device
 *     memory: callers size scratch with the *_bytes() queries and pass it in;
 *   - the return value is a knnag_status; KNNAG_OK means all kernels were
 *     enqueued.  Errors detected on the device (a bounded wait that gave up)
 *     are latched in a status word inside the caller's workspace and read
 *     back with knnag_read_device_status().
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the LemonATsu/CUDA-kNN-Aniso-Gaussian-Feature-Aggregation project).
 */
#ifndef KNN_ANISO_H_
#define KNN_ANISO_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  KNNAG_OK = 0,
  KNNAG_ERR_ARG = 1,        /* null pointer, negative or inconsistent size */
  KNNAG_ERR_K = 2,          /* K < 1 or K > P */
  KNNAG_ERR_DTYPE = 3,      /* dtype not KNNAG_F32 / KNNAG_F64 */
  KNNAG_ERR_WORKSPACE = 4,  /* workspace smaller than the *_bytes() query */
  KNNAG_ERR_TOO_LARGE = 5,  /* B*Q*K or B*P exceeds the 32-bit index range */
  KNNAG_ERR_CUDA = 6,       /* a launch failed (cudaGetLastError) */
  KNNAG_ERR_DEVICE = 7,     /* latched on the device: a bounded wait gave up, or a
                               segment table failed validation (ragged calls) */
  KNNAG_ERR_SCRATCH_LIMIT = 8 /* needs more than knnag_forward_noalloc's fixed scratch */
} knnag_status;

enum { KNNAG_F32 = 0, KNNAG_F64 = 1 };

/* Bits of the `needs` mask of the backward entry points: which outputs to
 * write.  Outputs whose bit is clear may be NULL. */
enum {
  KNNAG_NEED_DQ = 1,
  KNNAG_NEED_DP = 2,
  KNNAG_NEED_DF = 4,
  KNNAG_NEED_DSIGMA = 8,
  KNNAG_NEED_DR = 16,
  KNNAG_NEED_DGFO = 32,
  KNNAG_NEED_ALL = 63,
  /* Not an output: grad_f_out points to ONE value broadcast over [B,Q,F]
   * (the gradient of f_out.sum(), whose broadcast autograd does not
   * materialise).  The kernels then use a row sum of f instead of F-wide
   * dot products with grad_f_out rows, and write s * sum(w) to every
   * column of df, instead of gathering grad_f_out rows. */
  KNNAG_GFO_SCALAR = 64
};

/* Human-readable text of a status code (static storage). */
const char* knnag_status_string(int status);

/* Library version, as major*10000 + minor*100 + patch. */
int knnag_version(void);

/* ------------------------------------------------------------------ forward */

/* Bytes of scratch knnag_forward needs (256-byte aligned base expected). */
size_t knnag_forward_workspace_bytes(int B, int Q, int P, int F, int K, int dtype);

/*
 * Fused kNN search + weighted feature aggregation.
 * Replaces knn_aggregate_aniso_forward (csrc/knn_aggregate.cpp:26-47) and its
 * launcher knn_aggregate_aniso_forward_cuda (csrc/forward.cu:286-338) with the
 * kernel csrc/forward.cu:56-110 and csrc/mink.cuh.
 * Outputs: f_out [B,Q,F], w_out [B,Q,K], dists [B,Q,K] (dtype), idxs [B,Q,K]
 * int64.  Requires 1 <= K <= P.  `points` (optional, may be NULL) receives the
 * packed per-point records (knnag_points_bytes) that the backward entry
 * points can reuse instead of re-packing p, sigma and R.
 */
int knnag_forward(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                  int B, int Q, int P, int F, int K, int dtype,
                  void* f_out, void* w_out, void* dists, int64_t* idxs,
                  void* points, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Same result as knnag_forward, for callers that cannot allocate device
 * memory (allocator-free sections of a serving loop, plugins whose host
 * framework owns every device allocation): no workspace argument, no
 * allocation.  The scratch is one fixed 8 MiB device array inside the
 * library, held by every GPU that loads it until process exit; sizes whose
 * scratch would exceed it return KNNAG_ERR_SCRATCH_LIMIT (the scratch is
 * about 276 bytes per point plus 19 bytes per query: up to ~31k points with
 * few queries, or ~15k points with ~230k queries).  The first call on each device looks the
 * array's address up (cudaGetSymbolAddress) and should come before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race.  No counterpart in the reference.
 */
int knnag_forward_noalloc(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                          int B, int Q, int P, int F, int K, int dtype,
                          void* f_out, void* w_out, void* dists, int64_t* idxs, void* stream);

/* The device status word of knnag_forward_noalloc's fixed scratch on the
 * current device, read and cleared as knnag_read_device_status does for a
 * workspace (synchronises `stream`).  Read it after a call and before the
 * next one, which clears it.  The scratch address is cached per device for
 * the life of the device's primary context.  No counterpart in the
 * reference. */
int knnag_noalloc_read_device_status(void* stream);

/* ----------------------------------------------------- forward variants */

/* Bytes of scratch the variant entry points below need. */
size_t knnag_variant_workspace_bytes(int B, int Q, int P, int dtype);

/*
 * Aggregation at caller-given neighbour indices knn_idxs [B,Q,K] int64
 * (no search, no sorting): dists = key, w_out = exp(-key), f_out = sum_k
 * w_k f[idx_k].  Replaces knn_precomputed_aggregate_aniso_forward
 * (csrc/knn_aggregate.cpp:76-99, csrc/forward.cu:186-230, 398-450).  An index
 * outside [0, P) contributes nothing (w = 0, dist = +inf).
 */
int knnag_forward_precomputed(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                              const int64_t* knn_idxs, int B, int Q, int P, int F, int K, int dtype,
                              void* f_out, void* w_out, void* dists,
                              void* workspace, size_t workspace_bytes, void* stream);

/*
 * Lookup variant: the Euclidean nearest point of each query (strict '<'
 * scan, first index wins), then row `nearest` of knn_table [P, table_cols]
 * int64 (shared by all batch elements; its first K entries, in table order,
 * unsorted) with anisotropic weights.  Outputs as knnag_forward.
 * Replaces knn_lookup_aggregate_aniso_forward (csrc/knn_aggregate.cpp:50-73,
 * csrc/forward.cu:113-183, 341-395).
 */
int knnag_forward_lookup(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                         const int64_t* knn_table, int table_cols, int B, int Q, int P, int F, int K, int dtype,
                         void* f_out, void* w_out, void* dists, int64_t* idxs,
                         void* workspace, size_t workspace_bytes, void* stream);

/*
 * Isotropic forward: K nearest points by squared Euclidean distance (MinK
 * rules), w_k = exp(-d_k * sigma[idx_k][0]) with sigma [B,P,sigma_cols],
 * f_out = sum_k w_k f[idx_k], w_sum [B,Q,1] = sum_k w_k.  Replaces
 * knn_aggregate_forward (csrc/knn_aggregate.cpp:5-23, csrc/forward.cu:5-53,
 * 233-283).  Needs no workspace.
 */
int knnag_forward_isotropic(const void* q, const void* p, const void* f, const void* sigma, int sigma_cols,
                            int B, int Q, int P, int F, int K, int dtype,
                            void* f_out, void* w_sum, void* dists, int64_t* idxs, void* stream);

/* ---------------------------------------------------------- adjoint index */

/* Bytes of the packed per-point records (16 values of dtype per point).  A
 * points buffer must be 16-byte aligned (KNNAG_ERR_ARG otherwise). */
size_t knnag_points_bytes(int B, int P, int dtype);

/* Pack p, sigma and R into per-point records (what knnag_forward also writes). */
int knnag_pack_points(const void* p, const void* sigma, const void* R, int B, int P, int dtype,
                      void* points, void* stream);

/* Bytes of the point->entry adjacency (CSR) built by knnag_build_adjacency. */
size_t knnag_adjacency_bytes(int B, int Q, int P, int K);

/*
 * Inverse neighbour lists: for every point (b,i), the entries e = (b*Q+q)*K+k
 * with idxs[e] == i, in increasing e.  Deterministic.  `adjacency` holds
 * rowptr [B*P+1] int32 followed by the entry lists [B*Q*K] int32 and scratch.
 * No reference counterpart: the reference scatters with float atomicAdd
 * (csrc/backward.cu:91,102-119,291,308-326) instead.
 */
int knnag_build_adjacency(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, void* stream);

/*
 * knnag_forward that also makes the first pass of the point -> entry
 * adjacency: for every point (b, i) it counts the entries e with
 * idxs[e] == i into `adjacency` (knnag_adjacency_bytes(B, Q, P, K), 16-byte
 * aligned), as the entries are written; knnag_build_adjacency_counted on the
 * same buffer and idxs then skips that pass.  A caller that will need
 * point-side gradients (it wants dp, df, dsigma or dR) saves the counting
 * launch of the backward this way.  No reference counterpart.
 */
int knnag_forward_counted(const void* q, const void* p, const void* f, const void* sigma, const void* R,
                          int B, int Q, int P, int F, int K, int dtype,
                          void* f_out, void* w_out, void* dists, int64_t* idxs,
                          void* points, void* adjacency, void* workspace, size_t workspace_bytes, void* stream);

/* knnag_build_adjacency for a buffer whose per-point counts were written by
 * knnag_forward_counted with these idxs (and not used since). */
int knnag_build_adjacency_counted(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, void* stream);

/* --------------------------------------------------------------- backward */

/* Bytes of scratch knnag_backward / knnag_backward_2nd need. */
size_t knnag_backward_workspace_bytes(int B, int Q, int P, int F, int K, int dtype);

/*
 * First-order adjoint of f_out.
 * Replaces knn_aggregate_aniso_backward (csrc/knn_aggregate.cpp:101-132) and
 * knn_aggregate_aniso_backward_cuda (csrc/backward.cu:331-389, kernel
 * csrc/backward.cu:5-121).  grad_w_out is accepted and ignored, as in the
 * reference (csrc/backward.cu:93-94).  w_out may be NULL: weights are then
 * recomputed from idxs (bit-identical to the forward's).  points/adjacency
 * may be NULL: they are then built in the workspace.  coef_out (optional,
 * [B,Q,K] dtype) receives c = grad_f_out[q] . f[idx], reusable by
 * knnag_backward_2nd.  Outputs: dq [B,Q,3], dp [B,P,3], df [B,P,F],
 * dsigma [B,P,3], dR [B,P,3,3], each written in full when its `needs` bit is set.
 */
int knnag_backward(const void* grad_f_out, const void* grad_w_out,
                   const void* q, const void* p, const void* f, const void* sigma, const void* R,
                   const void* w_out, const int64_t* idxs,
                   int B, int Q, int P, int F, int K, int dtype, int needs,
                   const void* points, const void* adjacency,
                   void* dq, void* dp, void* df, void* dsigma, void* dR, void* coef_out,
                   void* workspace, size_t workspace_bytes, void* stream);

/*
 * Second-order adjoint through dL/dq (Eikonal): gradients of
 * <grad_grad_q, dq(grad_f_out)> w.r.t. grad_f_out, q, p, f, sigma and R.
 * Replaces knn_aggregate_aniso_backward_2nd (csrc/knn_aggregate.cpp:135-172)
 * and knn_aggregate_aniso_backward_2nd_cuda (csrc/backward.cu:392-455, kernel
 * csrc/backward.cu:124-328).  grad_w_out is ignored.  coef (optional) is the
 * coef_out of the matching knnag_backward call; NULL recomputes it.
 * Outputs: dgfo [B,Q,F], dq [B,Q,3], dp, df, dsigma, dR as above.
 */
int knnag_backward_2nd(const void* grad_grad_q, const void* grad_f_out, const void* grad_w_out,
                       const void* q, const void* p, const void* f, const void* sigma, const void* R,
                       const void* w_out, const int64_t* idxs,
                       int B, int Q, int P, int F, int K, int dtype, int needs,
                       const void* points, const void* adjacency, const void* coef,
                       void* dgfo, void* dq, void* dp, void* df, void* dsigma, void* dR,
                       void* workspace, size_t workspace_bytes, void* stream);

/* Copy the device status word latched in a forward/backward workspace to the
 * host (synchronises `stream`) and clear it; returns KNNAG_OK or KNNAG_ERR_DEVICE. */
int knnag_read_device_status(void* workspace, void* stream);

/* ------------------------------------------- ragged batches (FP32 only)
 *
 * No single reference entry point: the reference takes one uniform batch per
 * call, so a batch of clouds with different P, Q and K is a host loop over
 * knn_aggregate_aniso_forward (csrc/knn_aggregate.cpp:26-47), one call per
 * cloud.  These entry points serve such a batch -- or a stream of requests
 * against resident clouds -- in one launch sequence.
 *
 * Cloud set: C clouds with P[c] points, their p [sum P, 3], sigma
 * [sum P, 3], R [sum P, 3, 3] and features f [sum P, F] concatenated in
 * cloud order.  The cloud-set buffer (device, 256-byte aligned -- calls
 * reject one that is not 16-byte aligned with KNNAG_ERR_ARG --
 * knnag_cloudset_bytes) holds the packed records and the search index of
 * every cloud and describes itself; kernels need only its address. */

/* Bytes of a cloud set of C clouds with P[c] >= 1 points (host array); 0 if invalid. */
size_t knnag_cloudset_bytes(int C, const int* P);

/* Scratch bytes of knnag_cloudset_build. */
size_t knnag_cloudset_build_workspace_bytes(int C, const int* P);

/* Write the cloud set's header and cloud table (host -> device copy; the
 * call synchronises `stream`, so it cannot be captured).  Needed once per
 * buffer and size list. */
int knnag_cloudset_init(int C, const int* P, void* cloudset, size_t cloudset_bytes, void* stream);

/* Pack the clouds' records and build their search index (Hilbert order, sorted
 * tiles, tile key bounds) from p, sigma, R.  Kernels only (capturable); call
 * again whenever the geometry changes.  The buffer must have been set up by
 * knnag_cloudset_init with the same C and P. */
int knnag_cloudset_build(const float* p, const float* sigma, const float* R, int C, const int* P, void* cloudset,
                         size_t cloudset_bytes, void* workspace, size_t workspace_bytes, void* stream);

/* Segment table: nseg query sets; segment s has Q[s] queries against cloud
 * cloud[s] with K[s] neighbours (1 <= K[s] <= P of that cloud).  Its queries
 * are rows [q_off, q_off + Q[s]) of q [sum Q, 3] and f_out [sum Q, F] (q_off
 * = sum of the Q before it), its neighbours entries [e_off, e_off + Q[s] K[s])
 * of w_out, dists, idxs (e_off = sum of Q K before it), idxs being point
 * indices within the cloud.  knnag_segments_encode writes the table into a
 * HOST buffer of knnag_segments_bytes(nseg); the caller copies it to a
 * device buffer (256-byte aligned) before the call that uses it.  `splits`
 * (the search launch shape code, as for knnag_set_search_splits) must match the forward's.  want_grad
 * (NULL: every segment) marks the segments knnag_ragged_grad_q serves; they
 * must come first. */
size_t knnag_segments_bytes(int nseg);
int knnag_segments_encode(int nseg, const int* cloud, const int* Q, const int* K, const int* want_grad, int C,
                          const int* cloud_P, int splits, void* table, size_t table_bytes);

/* Scratch bytes of knnag_ragged_forward for tables of at most cap_segments
 * segments and cap_queries queries. */
size_t knnag_ragged_workspace_bytes(int cap_segments, long long cap_queries);

/* Forward of every segment: kNN under the segment's cloud's anisotropic
 * keys, MinK order and tie rules, w_out = exp(-dists), f_out = sum_k w_k
 * f[idx_k] -- per segment bit-identical to knnag_forward on that cloud and
 * query set.  Sizes are read from the device table, so a captured graph of
 * this call replays on any table within the capacities (cap_segments,
 * cap_queries, cap_entries = sum Q K, max_k >= every K, max_cloud_points >=
 * every cloud's P).  A table outside them latches KNNAG_ERR_DEVICE in the
 * workspace status word (knnag_read_device_status) and writes nothing. */
int knnag_ragged_forward(const void* cloudset, const void* segments, const float* q, const float* f, int F,
                         int cap_segments, long long cap_queries, long long cap_entries, int max_k,
                         int max_cloud_points, int splits, float* f_out, float* w_out, float* dists, int64_t* idxs,
                         void* workspace, size_t workspace_bytes, void* stream);

/* dq = d<grad_f_out, f_out>/dq of the segments marked want_grad (rows
 * [0, their total Q)) at the forward's idxs (weights recomputed; grad_f_out
 * NULL means all ones, i.e. d(sum f_out)/dq) -- the first-order query
 * gradient of knnag_backward.  With grad_f_out NULL, f_row_sums (optional,
 * [sum P], from knnag_feature_row_sums of f) replaces the F-wide dot
 * products by c = rowsum(f)[idx], bit-identical to what the uniform op's
 * backward of f_out.sum() computes.  workspace: 256 bytes (status word). */
int knnag_ragged_grad_q(const void* cloudset, const void* segments, const float* q, const float* f, int F,
                        const float* grad_f_out, const float* f_row_sums, const int64_t* idxs, int cap_segments,
                        long long cap_queries, long long cap_entries, int max_k, int max_cloud_points, float* dq,
                        void* workspace, size_t workspace_bytes, void* stream);

/* Per-row sums over the F columns of f [rows, F] (dtype) into out [rows],
 * in the fixed order the backward entry points use.  No reference
 * counterpart. */
int knnag_feature_row_sums(const void* f, long long rows, int F, int dtype, void* out, void* stream);

/* ---------------------------------------------------------- instrumentation
 * No reference counterpart (the reference has no timing hooks). */

/* Process-wide: when both are non-NULL (cudaEvent_t), every later
 * knnag_forward records ev_begin just before and ev_end just after its kNN
 * search kernel on the call's stream -- as external event nodes when the call
 * is captured into a CUDA graph -- so the search can be timed inside a larger
 * step.  Pass NULLs to switch off. */
void knnag_set_profile_events(void* ev_begin, void* ev_end);

/* Process-wide count of kernels this library has launched so far. */
long long knnag_launch_count(void);

/* Tuning: launch shape of the FP32 search of every later knnag_forward /
 * knnag_forward_noalloc in the process (the autotuner sets it from timings
 * cached per shape bucket): 1, 2, 4 -> CTAs of 4, 2, 1 warps of 32 queries;
 * 8 -> 2 warps of 16 queries; 16 -> 4 warps of 8 queries; 32 -> 1 warp of
 * 16; 64 -> 1 warp of 8 (fewer queries per warp give more warps for small
 * query sets); 128 -> the tensor-core filtered search (approximate keys of
 * 128 queries x 128 points per tcgen05 MMA, exact keys for the candidates);
 * 0 restores the automatic choice (the tensor-core search for grids of more
 * than 8 waves of its CTAs, else by the warps the query set gives).  Results
 * do not depend on it.  Returns KNNAG_ERR_ARG for other values.  Codes 1-64
 * are also the `splits` of segment tables.  No reference counterpart. */
int knnag_set_search_splits(int splits);
int knnag_get_search_splits(void);

/* Test hook of the search kernels' bounded waits (process-wide; affects
 * every later FP32 search launch).  visit >= 0: the tile copy of that
 * visit position of every search CTA is armed on its mbarrier but never
 * issued, so the waits on it give up after wait_spins sleeps of 256 ns
 * (0: the default budget, about a second), the kernel latches
 * KNNAG_ERR_DEVICE in the workspace status word and returns without writing
 * that CTA's outputs.  knnag_debug_set_search_stall(-1, 0) restores normal
 * operation.  Returns KNNAG_ERR_ARG for visit < -1 or wait_spins < 0.  No
 * reference counterpart (the reference has no bounded waits). */
int knnag_debug_set_search_stall(int visit, int wait_spins);

/* Launch an FFMA-bound kernel (blocks x 256 threads, `iters` iterations of 16
 * independent FMA chains per thread, 32*iters FLOP per thread) writing one
 * float per thread to `out`; used to measure the FP32 peak the search kernel
 * is compared against. */
int knnag_fp32_peak_probe(float* out, int blocks, int iters, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* KNN_ANISO_H_ */
