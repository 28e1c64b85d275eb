// Internal parameter blocks and workspace layout shared by the .cu files of
// libknn_aniso.so.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stddef.h>
#include <stdint.h>

#include "knn_ragged.h"

namespace knnag {

// NVTX range over one host-side stage of a call (the kernels it enqueues
// show up under it in a timeline profiler; without one attached the push
// and pop are no-ops).  Names start with "knnag:".
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

template <typename T>
struct ExactParams {
  const T* q;
  const T* rec;  // per-point records [B*P*16]
  const T* f;
  // isotropic forward only (key = squared Euclidean distance): raw points,
  // sigma [B,P,iso_stride] (component 0 scales the key in the weight); the
  // weight sum goes to w_out[B,Q,1]
  const T* iso_p;
  const T* iso_sigma;
  int iso_stride;
  int B, Q, P, F, K;
  int use_list;            // 1: process list[0 .. *list_count), 0: every query
  const int* list;
  const int* list_count;
  T* f_out;
  T* w_out;
  T* dists;
  int64_t* idxs;
  // ragged calls (FP32): per-query sizes and offsets from the segment table,
  // records from the cloud set.  List items are global query rows; without a
  // list the kernel serves the queries of segments with K > 32.  Nothing is
  // done when *status is nonzero (a table that failed validation); a list
  // row out of range latches kStatusBadIndex there.
  const char* cs;
  const void* segs;
  int* status;
  // optional (uniform calls): per point row b*P + i, the number of written
  // entries that select it (the adjacency's first pass), zeroed beforehand
  int* adj_count;
};

struct SearchParams {
  const float* q;
  const int* perm_q;   // sorted position -> query index, per batch element
  const float* tinfo;  // per tile kTinfoFloats: its box and its sub-boxes (box, mu, pad)
  int ntile;           // tiles per batch element (ragged: the most of any cloud)
  const float* pairs;  // pair-interleaved tiles [B][P_pad/2][32]
  const float* rec;    // per-point records [B*P*16]
  const float* f;
  int B, Q, P, P_pad, F, K;
  int vec4;            // f and f_out rows may be read/written as float4
  float* f_out;
  float* w_out;
  float* dists;
  int64_t* idxs;
  int* status;
  int* flag_count;
  int* flag_list;      // flagged queries: global query rows
  // ragged calls: records, tiles and boxes come from the cloud set, sizes
  // and offsets from the segment table; work items are taken in order from
  // item_counter
  const char* cs;
  const void* segs;
  int* item_counter;
  // Test hook of the timeout path (knnag_debug_set_search_stall): the tile
  // copy of visit `stall_visit` is armed on its mbarrier but never issued,
  // so the waits on it run out after `wait_spins` sleeps; -1 (no stall)
  // and the default budget otherwise.
  int stall_visit;
  int wait_spins;
  // optional (uniform calls): entries per point row, counted as written
  int* adj_count;
  // optional (uniform calls): per batch element [Q], sorted query position
  // -> a position in the sorted point order near the query (the middle of
  // its cell's points), where the seed window of the threshold is taken
  const int* qseed;
  // optional (uniform calls): the plan kernels' outputs, read by the search:
  // seed thresholds per sorted query [B*Q], the CTA items (batch element,
  // first and end sorted query, 0), and the per-block estimates
  float* tau0;
  int4* items;
  int* plan_est;
  // tensor-core filtered search (uniform calls): per tile the B operand of
  // the approximate-key GEMM [B*ntile][kTcOpsFloats] and its error-bound
  // terms [B*ntile][kTcInfoFloats], written by the tile-info kernel
  const float* tcops;
  const float* tcinfo;
};

// Search CTA: WPC warps (1, 2 or 4), each owning QPW queries (32, 16 or 8;
// lane j < QPW keeps query j's list) and sharing the CTA's tile ring; a work
// item is the CTA's WPC * QPW queries.  The C ABI's launch-shape code s
// (knnag_set_search_splits, the segment tables' `splits`) selects
//   s = 1: 4 warps x 32    s = 2: 2 x 32    s = 4: 1 x 32
//   s = 8: 2 warps x 16    s = 16: 4 x 8    s = 32: 1 x 16    s = 64: 1 x 8
// i.e. 128, 64, 32, 32, 32, 16 and 8 queries per CTA.
constexpr int kSearchMaxThreads = 128;
// Candidate queue entries per query: 64 points (the points a query meets
// between two folds of its queue) always fit.
constexpr int kQCap = 64;
// Tile buffers of the search ring: visit v lands in buffer v % kTileBufs,
// so kTileBufs - 1 copies are in flight while a tile is being read.
constexpr int kTileBufs = 2;
constexpr size_t kSearchTileBytes = 8192;  // 128 points x 16 floats
static_assert(kTileBufs * 12 + 8 <= 64, "search ring bookkeeping exceeds its 64 bytes");
__host__ __device__ inline constexpr int search_wpc(int shape) {
  return shape == 1 ? 4 : shape == 2 ? 2 : shape == 4 ? 1 : shape == 8 ? 2 : shape == 16 ? 4 : 1;
}
__host__ __device__ inline constexpr int search_qpw(int shape) {
  return shape <= 4 ? 32 : (shape == 8 || shape == 32) ? 16 : 8;
}
__host__ __device__ inline constexpr int search_qpc(int shape) { return search_wpc(shape) * search_qpw(shape); }
inline bool search_shape_ok(int shape) {
  return shape == 1 || shape == 2 || shape == 4 || shape == 8 || shape == 16 || shape == 32 || shape == 64;
}
// Launch-shape code of the uniform search that filters candidates with
// approximate keys from the tensor cores (search_tc_kernel: 128 queries per
// CTA, one thread per query); uniform calls only (segment tables take the
// codes above).
constexpr int kShapeTensorFilter = 128;
inline bool search_setting_ok(int shape) { return search_shape_ok(shape) || shape == kShapeTensorFilter; }

// Shared-memory layout of the search kernel with `wpc` warps of `qpw` queries:
//   ring      kTileBufs tiles
//   queues    wpc x [qpw queries][kQCap] keys, then indices (after the tile
//             loop: the CTA's sorted lists, weights and flags)
//   qtab      [wpc qpw] float4 (x, y, z, threshold) of the CTA's queries
//   ctab      per warp, the queries a pass matters to, compacted: [qpw]
//             float4 (x, y, z, threshold) of the warp, then [qpw] their lanes
//   tring     kTileBufs tile infos (box and sub-boxes), copied with the tiles
//   misc      [wpc qpw] original query index, [wpc][6] warp query boxes,
//             64 bytes of mbarriers / counters / flags
//   region C  tile bounds and visit order [NTP x 8 B] + visit counter
__host__ __device__ inline constexpr size_t search_queue_off() { return (size_t)kTileBufs * kSearchTileBytes; }
__host__ __device__ inline constexpr size_t search_warp_queue_bytes(int qpw) { return (size_t)qpw * kQCap * 8; }
__host__ __device__ inline constexpr size_t search_qtab_off(int wpc, int qpw) {
  return search_queue_off() + (size_t)wpc * search_warp_queue_bytes(qpw);
}
__host__ __device__ inline constexpr size_t search_ctab_off(int wpc, int qpw) {
  return search_qtab_off(wpc, qpw) + (size_t)wpc * qpw * 16;
}
__host__ __device__ inline constexpr size_t search_tring_off(int wpc, int qpw) {
  return search_ctab_off(wpc, qpw) + (size_t)wpc * qpw * 20;
}
__host__ __device__ inline constexpr size_t search_misc_off(int wpc, int qpw) {
  return search_tring_off(wpc, qpw) + (size_t)kTileBufs * kTinfoBytes;
}
__host__ __device__ inline constexpr size_t search_bars_off(int wpc, int qpw) {
  return search_misc_off(wpc, qpw) + (size_t)wpc * qpw * 4 + (size_t)wpc * 6 * 4;
}
__host__ __device__ inline constexpr size_t search_smem_bytes(int wpc, int qpw) { return search_bars_off(wpc, qpw) + 64; }
// Tiles per cloud rounded up to a power of two (the visit-order sort).
__host__ __device__ inline int search_tiles_pow2(int ntile) {
  int n = 1;
  while (n < ntile) n <<= 1;
  return n;
}
__host__ __device__ inline size_t search_region_c_bytes(int ntile) { return (size_t)search_tiles_pow2(ntile) * 8 + 16; }
// The sorted lists of a query (keys, indices, weights) and its flag, staged
// for the epilogue, must fit the query's share of the queue region.
static_assert((size_t)33 * 12 + 4 <= (size_t)kQCap * 8, "epilogue staging exceeds the queue region");

// ------------------------------------------------------------- workspace
// Forward workspace: [status, flag_count] | flag_list [B*Q] | records (when
// the caller passed no points buffer) | pair tiles (FP32 fast path).
struct FwdLayout {
  size_t status, flag_list, rec, pairs, total;
  // spatial index (FP32 search path): bound parts [B*kBoundParts*8], cell counts / offsets
  // [B*cells(+1)], point and query permutations, tile boxes [B*ntile*8]
  size_t bounds, cell_count, cell_offset, perm_p, perm_q, tinfo;
  size_t qseed;  // [B*Q] ints: seed positions of the sorted queries
  size_t tau0, plan_est, items;  // search plan: seeds [B*Q], estimates, CTA items
  size_t tcops, tcinfo;          // tensor-core filter: per tile B operand and bound terms
  int P_pad, bits;
};
int spatial_bits(int P);
// tc_ops: also write the tensor-core filter's per-tile operands (L.tcops, L.tcinfo)
int launch_spatial_index(const float* q, const float* rec, int B, int Q, int P, int P_pad, char* ws, const FwdLayout& L,
                         cudaStream_t st, bool tc_ops = false);
int launch_exclusive_scan(int* count, int n, int* out, cudaStream_t st);
int launch_cloudset_index(char* cs, const CloudSetHeader& h, const CloudDesc* cd_dev, int max_p, int max_ntile,
                          int* cnt, int* perm_p, cudaStream_t st);
int launch_query_order(const float* q, const char* cs, const void* segs_dev, int cap_segs, int64_t cap_q,
                       int cap_cells, int* cnt, int* off, int* perm_q, const int* status, cudaStream_t st);

// Ragged forward workspace: [status, flag_count, item_counter] | flag_list
// [cap_q] | perm_q [cap_q] | query cell counts / offsets [cap_cells (+1)],
// cap_cells = cap_q + 8 * cap_segs (a segment of Q queries has at most
// max(Q, 8) cells).
struct RaggedLayout {
  size_t status, flag_list, perm_q, cell_count, cell_offset, total;
  int64_t cap_cells;
};
RaggedLayout ragged_layout(int cap_segs, int64_t cap_q);
int launch_validate_segments(const char* cs, const void* segs, int cap_segs, int64_t cap_q, int64_t cap_e, int max_k,
                             int ntile_cap, int qpc, int* status, cudaStream_t st);
int ragged_forward_impl(const char* cs, const void* segs, const float* q, const float* f, int F, int cap_segs,
                        int64_t cap_q, int64_t cap_e, int max_k, int ntile_cap, int splits, float* f_out, float* w_out,
                        float* dists, int64_t* idxs, void* workspace, cudaStream_t st);
int ragged_grad_q_impl(const char* cs, const void* segs, const float* q, const float* f, int F, const float* gfo,
                       const float* f_row_sums, const int64_t* idxs, int64_t cap_q, float* dq, const int* status,
                       cudaStream_t st);
int launch_row_sums(const void* f, int64_t rows, int F, int dtype, void* out, cudaStream_t st);
template <typename T>
int launch_exact(const ExactParams<T>& a, cudaStream_t st);
int variants_precomputed(const void* q, const void* f, const void* rec, const int64_t* idxs, int B, int Q, int P,
                         int F, int K, int dtype, void* f_out, void* w_out, void* dists, cudaStream_t st);
int variants_lookup(const void* q, const void* p, const void* f, const void* rec, const int64_t* table, int tstride, int B, int Q,
                    int P, int F, int K, int dtype, int* nearest, void* f_out, void* w_out, void* dists,
                    int64_t* idxs, cudaStream_t st);
FwdLayout fwd_layout(int B, int Q, int P, int K, int dtype, bool own_rec);

// Adjacency (CSR) layout: rowptr [B*P+1] | cursor [B*P] | unsorted [N] | entries [N].
struct AdjLayout {
  size_t rowptr, cursor, unsorted, entries, total;
};
AdjLayout adj_layout(int B, int Q, int P, int K);

// Tensor-core filtered search of a uniform FP32 call (knn_search_tc.cu);
// KNNAG_ERR_TOO_LARGE when its shared memory does not fit (the caller then
// takes the CUDA-core search).
int launch_search_tc(const SearchParams& a, cudaStream_t st);
// Whether the tensor-core search's shared memory fits for `ntile` tiles.
bool search_tc_fits(int ntile);
// The search plan (knn_search.cu) for blocks of qpc sorted queries, nb per
// batch element: seed thresholds into a.tau0, the blocks' estimates into
// a.plan_est, the CTA items, heaviest first, into a.items.
int launch_search_plan(const SearchParams& a, int qpc, int nb, cudaStream_t st);
// Most blocks the plan orders (its estimates are staged in shared memory).
int search_plan_max_blocks();
int num_sms(int dev);

// Process-wide split count of the uniform search (0: automatic), set by
// knnag_set_search_splits (defined in knn_capi.cu).
int search_splits_setting();
// Process-wide test hook of the search's bounded waits, set by
// knnag_debug_set_search_stall (defined in knn_capi.cu): writes the
// stall_visit / wait_spins fields of a SearchParams.
void apply_search_debug(SearchParams& sp);

// Instrumentation shared by the .cu files (defined in knn_capi.cu).
void note_launches(int n);
void profile_begin(cudaStream_t st);
void profile_end(cudaStream_t st);

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Backward workspace: status | records | adjacency | per-entry coefficients.
struct BwdLayout {
  size_t status, rec, adj, coef, rowsum, total;  // rowsum: sum over columns of f per point (scalar grad_f_out)
};
BwdLayout bwd_layout(int B, int Q, int P, int F, int K, int dtype);

// Arguments of one backward call (order 1 or 2).
struct BwdArgs {
  int order;
  const void *ggq, *gfo, *q, *p, *f, *sigma, *R, *w_in;
  const int64_t* idxs;
  int B, Q, P, F, K, dtype, needs;
  const void *points, *adjacency, *coef_in;
  void *dgfo, *dq, *dp, *df, *dsigma, *dR, *coef_out;
  void* workspace;
};
int backward_impl(const BwdArgs& x, cudaStream_t st);

// Packs the point records; block 0 also zeroes zero_words[0..n_zero) (a
// call's status words) so no separate memset is needed.
int launch_pack_points(const void* p, const void* sigma, const void* R, int B, int P, int dtype, void* rec,
                       cudaStream_t st, int* zero_words = nullptr, int n_zero = 0, int* zero_rows = nullptr);
// Chunks per batch element of the FP32 packing kernel that also bounds the
// points: chunk c of element b writes its box to parts[(b * kBoundParts +
// c) * 8 ...] (min xyz, max xyz), which the cell kernels reduce.
constexpr int kBoundParts = 32;
int launch_pack_points_bounded(const float* p, const float* sigma, const float* R, int B, int P, float* rec,
                               float* parts, cudaStream_t st, int* zero_words, int n_zero, int* zero_rows,
                               int* zero_cells, int64_t n_cells);
// adjacency: optional buffer (adj_layout) whose per-point entry counts the
// forward writes, for launch_build_adjacency(..., counted = true)
int forward_impl(const void* q, const void* p, const void* f, const void* sigma, const void* R, int B, int Q,
                 int P, int F, int K, int dtype, void* f_out, void* w_out, void* dists, int64_t* idxs,
                 void* points, void* workspace, cudaStream_t st, void* adjacency = nullptr);
int launch_build_adjacency(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, cudaStream_t st,
                           bool counted = false);

}  // namespace knnag
