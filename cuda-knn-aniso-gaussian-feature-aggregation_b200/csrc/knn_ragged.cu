// Ragged batches: cloud-set layout and build, segment-table encoding and
// validation, and the C ABI of the ragged forward and grad_q.
//
// The reference takes one uniform batch [B, Q|P, ...] per call
// (csrc/knn_aggregate.cpp:26-47); a ragged batch of clouds with different
// P, Q and K there is a host loop of such calls, one per cloud.  Here the
// whole batch is one call whose kernels read sizes and offsets from device
// tables, so it is one launch sequence (and one CUDA graph) however many
// clouds it holds.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "knn_aniso.h"
#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {
namespace {

constexpr int64_t kI32Max = 2147483647;

// Host layout of a cloud set; fills descs (C entries) when given.
size_t cloudset_layout(int C, const int* P, CloudSetHeader* h, CloudDesc* descs) {
  if (C < 1 || !P) return 0;
  int64_t total_p = 0, total_tiles = 0, total_cells = 0;
  int max_ntile = 0;
  for (int c = 0; c < C; ++c) {
    if (P[c] < 1) return 0;
    const int bits = spatial_bits(P[c]);
    const int ntile = (int)((P[c] + kTilePoints - 1) / kTilePoints);
    if (descs) descs[c] = CloudDesc{total_p, total_tiles, P[c], ntile, bits, (int)total_cells};
    total_p += P[c];
    total_tiles += ntile;
    total_cells += (int64_t)1 << (3 * bits);
    if (ntile > max_ntile) max_ntile = ntile;
    if (total_p > kI32Max / kRecLen || total_cells > kI32Max - 1) return 0;
  }
  CloudSetHeader x{};
  x.magic = kCloudSetMagic;
  x.C = C;
  x.max_ntile = max_ntile;
  x.total_cells = (int)total_cells;
  x.total_p = total_p;
  x.total_tiles = total_tiles;
  x.desc_off = 256;
  x.rec_off = (int64_t)align256(256 + (size_t)C * sizeof(CloudDesc));
  x.pairs_off = x.rec_off + (int64_t)align256((size_t)total_p * kRecLen * 4);
  x.tinfo_off = x.pairs_off + (int64_t)align256((size_t)total_tiles * kTilePoints * kRecLen * 4);
  x.bnd_off = x.tinfo_off + (int64_t)align256((size_t)total_tiles * kTinfoBytes);
  x.celloff_off = x.bnd_off + (int64_t)align256((size_t)C * 8 * 4);
  x.total_bytes = x.celloff_off + (int64_t)align256(((size_t)total_cells + 1) * 4);
  if (h) *h = x;
  return (size_t)x.total_bytes;
}

// Cloud-set build scratch: cell counts, point permutation (the cell offsets
// live in the cloud set).
struct BuildScratch {
  size_t cnt, perm, total;
};
BuildScratch build_scratch(const CloudSetHeader& h) {
  BuildScratch b{};
  b.cnt = 0;
  b.perm = align256((size_t)h.total_cells * 4);
  b.total = b.perm + align256((size_t)h.total_p * 4);
  return b;
}

// One thread per segment: every entry must lie inside the capacities the
// launches were sized for and inside its cloud, and the running offsets
// must be the prefix sums the encoder writes.  Any mismatch latches
// kStatusBadTable and every later ragged kernel of the call does nothing.
__global__ void validate_segments_kernel(const char* cs, const void* segs, int cap_segs, int64_t cap_q, int64_t cap_e,
                                         int max_k, int ntile_cap, int qpc, int64_t cap_cells, int* status) {
  const SegHeader* sh = static_cast<const SegHeader*>(segs);
  const CloudSetHeader* ch = reinterpret_cast<const CloudSetHeader*>(cs);
  __shared__ int bad;
  if (qpc <= 0) qpc = sh->qpc;  // any encoding (callers that use no work items)
  if (threadIdx.x == 0) {
    bad = (sh->magic != kSegMagic || ch->magic != kCloudSetMagic || sh->nseg < 1 || sh->nseg > cap_segs ||
           sh->total_q < 0 || sh->total_q > cap_q || sh->total_e < 0 || sh->total_e > cap_e || sh->kmax > max_k ||
           sh->qpc != qpc || (qpc != 8 && qpc != 16 && qpc != 32 && qpc != 64 && qpc != 128) || sh->total_qcells < 0 ||
           sh->total_qcells > cap_cells || sh->n_items < 0 || sh->bigk_q < 0 || sh->bigk_q > sh->total_q ||
           sh->grad_rows < 0 || sh->grad_rows > sh->total_q)
              ? 1
              : 0;
  }
  __syncthreads();
  if (!bad) {
    const SegDesc* sd = seg_descs(segs);
    const CloudDesc* cd = cloud_descs(cs);
    const int n = sh->nseg;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
      const SegDesc g = sd[s];
      bool ok = g.cloud >= 0 && g.cloud < ch->C && g.Q >= 0 && g.K >= 1 && g.K <= max_k && g.qbits >= 1 &&
                g.qbits <= 10;
      if (ok) {
        const CloudDesc c = cd[g.cloud];
        const int64_t items = g.K > 32 ? 0 : (g.Q + qpc - 1) / qpc;
        const int64_t bigk = g.K > 32 ? g.Q : 0;
        const int64_t cells = (int64_t)1 << (3 * g.qbits);
        ok = g.K <= c.P && c.ntile <= ntile_cap && g.q_off >= 0 && g.q_off + g.Q <= sh->total_q && g.e_off >= 0 &&
             g.e_off + (int64_t)g.Q * g.K <= sh->total_e && g.item_off >= 0 && g.item_off + items <= sh->n_items &&
             g.bigk_off >= 0 && g.bigk_off + bigk <= sh->bigk_q && g.qcell_off >= 0 &&
             g.qcell_off + cells <= sh->total_qcells;
        if (ok && s + 1 < n) {
          const SegDesc h = sd[s + 1];
          ok = h.q_off == g.q_off + g.Q && h.e_off == g.e_off + (int64_t)g.Q * g.K &&
               h.item_off == g.item_off + items && h.bigk_off == g.bigk_off + bigk &&
               h.qcell_off == g.qcell_off + cells;
        }
        if (ok && s == 0) ok = g.q_off == 0 && g.e_off == 0 && g.item_off == 0 && g.bigk_off == 0 && g.qcell_off == 0;
      }
      if (!ok) atomicOr(&bad, 1);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && bad) atomicOr(status, kStatusBadTable);
}

int qpc_of(int splits) { return search_shape_ok(splits) ? search_qpc(splits) : 0; }

}  // namespace

int launch_validate_segments(const char* cs, const void* segs, int cap_segs, int64_t cap_q, int64_t cap_e, int max_k,
                             int ntile_cap, int qpc, int* status, cudaStream_t st) {
  validate_segments_kernel<<<1, 256, 0, st>>>(cs, segs, cap_segs, cap_q, cap_e, max_k, ntile_cap, qpc,
                                              ragged_layout(cap_segs, cap_q).cap_cells, status);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

}  // namespace knnag

using namespace knnag;

extern "C" {

size_t knnag_cloudset_bytes(int C, const int* P) { return cloudset_layout(C, P, nullptr, nullptr); }

size_t knnag_cloudset_build_workspace_bytes(int C, const int* P) {
  CloudSetHeader h{};
  if (!cloudset_layout(C, P, &h, nullptr)) return 0;
  return build_scratch(h).total;
}

int knnag_cloudset_init(int C, const int* P, void* cloudset, size_t cloudset_bytes, void* stream) {
  if (!cloudset || !P || C < 1) return KNNAG_ERR_ARG;
  if ((uintptr_t)cloudset & 15u) return KNNAG_ERR_ARG;  // records and tiles are read with 16-byte loads
  CloudSetHeader h{};
  std::vector<CloudDesc> d((size_t)C);
  const size_t need = cloudset_layout(C, P, &h, d.data());
  if (!need) return KNNAG_ERR_TOO_LARGE;
  if (cloudset_bytes < need || ((uintptr_t)cloudset & 255u)) return KNNAG_ERR_WORKSPACE;
  std::vector<char> host((size_t)h.rec_off, 0);
  memcpy(host.data(), &h, sizeof(h));
  memcpy(host.data() + h.desc_off, d.data(), d.size() * sizeof(CloudDesc));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(cloudset, host.data(), host.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return KNNAG_ERR_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

int knnag_cloudset_build(const float* p, const float* sigma, const float* R, int C, const int* P, void* cloudset,
                         size_t cloudset_bytes, void* workspace, size_t workspace_bytes, void* stream) {
  if (!p || !sigma || !R || !cloudset || !workspace || !P || C < 1) return KNNAG_ERR_ARG;
  if ((uintptr_t)cloudset & 15u) return KNNAG_ERR_ARG;  // records and tiles are read with 16-byte loads
  CloudSetHeader h{};
  const size_t need = cloudset_layout(C, P, &h, nullptr);
  if (!need) return KNNAG_ERR_TOO_LARGE;
  if (cloudset_bytes < need || ((uintptr_t)cloudset & 255u)) return KNNAG_ERR_WORKSPACE;
  const BuildScratch b = build_scratch(h);
  if (workspace_bytes < b.total || ((uintptr_t)workspace & 15u)) return KNNAG_ERR_WORKSPACE;
  int max_p = 0;
  for (int c = 0; c < C; ++c) max_p = P[c] > max_p ? P[c] : max_p;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* cs = static_cast<char*>(cloudset);
  char* ws = static_cast<char*>(workspace);
  int rc = launch_pack_points(p, sigma, R, 1, (int)h.total_p, KNNAG_F32, cs + h.rec_off, st);
  if (rc) return rc;
  return launch_cloudset_index(cs, h, reinterpret_cast<const CloudDesc*>(cs + h.desc_off), max_p, h.max_ntile,
                               reinterpret_cast<int*>(ws + b.cnt), reinterpret_cast<int*>(ws + b.perm), st);
}

size_t knnag_segments_bytes(int nseg) {
  return nseg < 1 ? 0 : sizeof(SegHeader) + (size_t)nseg * sizeof(SegDesc);
}

int knnag_segments_encode(int nseg, const int* cloud, const int* Q, const int* K, const int* want_grad, int C,
                          const int* cloud_P, int splits, void* table, size_t table_bytes) {
  if (nseg < 1 || !cloud || !Q || !K || C < 1 || !cloud_P || !table) return KNNAG_ERR_ARG;
  bool grad_prefix = true;
  const int qpc = qpc_of(splits);
  if (!qpc) return KNNAG_ERR_ARG;
  if (table_bytes < knnag_segments_bytes(nseg)) return KNNAG_ERR_WORKSPACE;
  SegHeader h{};
  h.magic = kSegMagic;
  h.nseg = nseg;
  h.qpc = qpc;
  int64_t items = 0, cells = 0;
  SegDesc* sd = reinterpret_cast<SegDesc*>(static_cast<char*>(table) + sizeof(SegHeader));
  for (int s = 0; s < nseg; ++s) {
    if (cloud[s] < 0 || cloud[s] >= C || Q[s] < 0) return KNNAG_ERR_ARG;
    if (K[s] < 1 || K[s] > cloud_P[cloud[s]]) return KNNAG_ERR_K;
    if (want_grad) {
      if (want_grad[s] && !grad_prefix) return KNNAG_ERR_ARG;  // segments wanting dq must come first
      if (!want_grad[s]) grad_prefix = false;
      else h.grad_rows += Q[s];
    }
    SegDesc g{};
    g.q_off = h.total_q;
    g.e_off = h.total_e;
    g.bigk_off = h.bigk_q;
    g.cloud = cloud[s];
    g.Q = Q[s];
    g.K = K[s];
    g.qbits = spatial_bits(Q[s] > 1 ? Q[s] : 1);
    g.qcell_off = (int)cells;
    g.item_off = (int)items;
    sd[s] = g;
    h.total_q += Q[s];
    h.total_e += (int64_t)Q[s] * K[s];
    if (K[s] > 32)
      h.bigk_q += Q[s];
    else
      items += (Q[s] + qpc - 1) / qpc;
    cells += (int64_t)1 << (3 * g.qbits);
    if (K[s] > h.kmax) h.kmax = K[s];
    if (h.total_q > kI32Max || items > kI32Max || cells > kI32Max - 1) return KNNAG_ERR_TOO_LARGE;
  }
  h.n_items = (int)items;
  h.total_qcells = (int)cells;
  if (!want_grad) h.grad_rows = h.total_q;
  memcpy(table, &h, sizeof(h));
  return KNNAG_OK;
}

size_t knnag_ragged_workspace_bytes(int cap_segments, long long cap_queries) {
  if (cap_segments < 1 || cap_queries < 0) return 0;
  return ragged_layout(cap_segments, cap_queries).total;
}

int knnag_ragged_forward(const void* cloudset, const void* segments, const float* q, const float* f, int F,
                         int cap_segments, long long cap_queries, long long cap_entries, int max_k,
                         int max_cloud_points, int splits, float* f_out, float* w_out, float* dists, int64_t* idxs,
                         void* workspace, size_t workspace_bytes, void* stream) {
  if (!cloudset || !segments || !f || !f_out || !w_out || !dists || !idxs || !workspace) return KNNAG_ERR_ARG;
  if ((uintptr_t)cloudset & 15u) return KNNAG_ERR_ARG;  // records and tiles are read with 16-byte loads
  if (cap_segments < 1 || cap_queries < 1 || cap_entries < 1 || F < 0 || max_cloud_points < 1) return KNNAG_ERR_ARG;
  if ((!q && cap_queries > 0) || !qpc_of(splits)) return KNNAG_ERR_ARG;
  if (max_k < 1 || max_k > max_cloud_points) return KNNAG_ERR_K;
  if (cap_queries > kI32Max / 2 || cap_segments > (1 << 24)) return KNNAG_ERR_TOO_LARGE;
  const RaggedLayout L = ragged_layout(cap_segments, cap_queries);
  if (workspace_bytes < L.total || ((uintptr_t)workspace & 15u)) return KNNAG_ERR_WORKSPACE;
  const int ntile_cap = (max_cloud_points + kTilePoints - 1) / kTilePoints;
  return ragged_forward_impl(static_cast<const char*>(cloudset), segments, q, f, F, cap_segments, cap_queries,
                             cap_entries, max_k, ntile_cap, splits, f_out, w_out, dists, idxs, workspace,
                             static_cast<cudaStream_t>(stream));
}

int knnag_ragged_grad_q(const void* cloudset, const void* segments, const float* q, const float* f, int F,
                        const float* grad_f_out, const float* f_row_sums, const int64_t* idxs, int cap_segments,
                        long long cap_queries, long long cap_entries, int max_k, int max_cloud_points, float* dq,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (!cloudset || !segments || !q || !f || !idxs || !dq || !workspace) return KNNAG_ERR_ARG;
  if ((uintptr_t)cloudset & 15u) return KNNAG_ERR_ARG;  // records and tiles are read with 16-byte loads
  if (cap_segments < 1 || cap_queries < 1 || cap_entries < 1 || F < 0 || max_cloud_points < 1) return KNNAG_ERR_ARG;
  if (max_k < 1 || max_k > max_cloud_points) return KNNAG_ERR_K;
  if (cap_queries > kI32Max / 2 || cap_segments > (1 << 24)) return KNNAG_ERR_TOO_LARGE;
  if (workspace_bytes < 256 || ((uintptr_t)workspace & 15u)) return KNNAG_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* status = static_cast<int*>(workspace);
  if (cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess) return KNNAG_ERR_CUDA;
  const int ntile_cap = (max_cloud_points + kTilePoints - 1) / kTilePoints;
  // qpc 0: any encoding is accepted (grad_q uses no search work items)
  int rc = launch_validate_segments(static_cast<const char*>(cloudset), segments, cap_segments, cap_queries,
                                    cap_entries, max_k, ntile_cap, 0, status, st);
  if (rc) return rc;
  return ragged_grad_q_impl(static_cast<const char*>(cloudset), segments, q, f, F, grad_f_out, f_row_sums, idxs,
                            cap_queries, dq, status, st);
}

int knnag_feature_row_sums(const void* f, long long rows, int F, int dtype, void* out, void* stream) {
  if (!f || !out || rows < 0 || F < 1) return KNNAG_ERR_ARG;
  if (dtype != KNNAG_F32 && dtype != KNNAG_F64) return KNNAG_ERR_DTYPE;
  if (rows == 0) return KNNAG_OK;
  return launch_row_sums(f, rows, F, dtype, out, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
