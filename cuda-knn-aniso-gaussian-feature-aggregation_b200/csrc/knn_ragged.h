// Ragged batches: resident cloud sets and segment tables (internal).
//
// A cloud set holds C point clouds of different sizes in one device buffer
// that describes itself: a header, one CloudDesc per cloud, then the packed
// point records, the Hilbert-sorted search tiles, the tile boxes and the
// per-cloud bounds of all clouds back to back.  Kernels find every region
// from the header, so the host needs only the buffer's address.
//
// A segment table lists the query sets of one ragged call: segment s has
// Q_s queries (rows [q_off, q_off + Q_s) of q and f_out) against cloud
// `cloud` with K_s neighbours (entries [e_off, e_off + Q_s*K_s) of dists,
// w_out and idxs; idxs are point indices within the cloud).  The table is
// encoded on the host (knnag_segments_encode) and copied to the device by
// the caller, so a captured CUDA graph can be replayed on new tables of the
// same capacity: every kernel reads the live counts from the device copy.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace knnag {

constexpr uint32_t kCloudSetMagic = 0x4b4e4353u;  // "SCNK"
constexpr uint32_t kSegMagic = 0x4b4e5347u;       // "GSNK"

struct CloudDesc {
  int64_t p_off;    // first point of the cloud (rows of p, f, records)
  int64_t tile_off; // first search tile of the cloud (128 points per tile)
  int P, ntile, bits, cell_off;  // cell_off: offset of the cloud's grid cells
};

struct CloudSetHeader {
  uint32_t magic;
  int C, max_ntile, total_cells;
  int64_t total_p, total_tiles;
  int64_t desc_off, rec_off, pairs_off, tinfo_off, bnd_off, total_bytes;
  // exclusive scan of the point counts of every cloud's grid cells
  // [total_cells + 1] (global point positions): where a query's cell starts
  // in its cloud's sorted points, for the search's seed windows
  int64_t celloff_off;
};

struct SegDesc {
  int64_t q_off;    // first query row
  int64_t e_off;    // first neighbour entry
  int64_t bigk_off; // first row among the queries of segments with K > 32
  int cloud, Q, K, qbits;
  int qcell_off;    // offset of the segment's query grid cells
  int item_off;     // first search work item (queries per item = qpc)
};

struct SegHeader {
  uint32_t magic;
  int nseg, kmax, qpc;
  int64_t total_q, total_e;
  int n_items, total_qcells;
  int64_t bigk_q;   // queries in segments with K > 32 (served by the exact kernel)
  int64_t grad_rows;  // rows [0, grad_rows) get dq from knnag_ragged_grad_q
  int64_t reserved;   // (header = 64 bytes; the SegDesc array follows)
};
static_assert(sizeof(SegHeader) == 64 && sizeof(SegDesc) == 48 && sizeof(CloudDesc) == 32, "table layout");

__host__ __device__ inline const CloudDesc* cloud_descs(const void* cs) {
  const CloudSetHeader* h = static_cast<const CloudSetHeader*>(cs);
  return reinterpret_cast<const CloudDesc*>(static_cast<const char*>(cs) + h->desc_off);
}
__host__ __device__ inline const SegDesc* seg_descs(const void* st) {
  return reinterpret_cast<const SegDesc*>(static_cast<const char*>(st) + sizeof(SegHeader));
}

// Last segment s with key(s) <= x (segments are in ascending key order; an
// empty segment shares its key with the next one and is skipped this way).
template <typename KeyFn>
__device__ __forceinline__ int seg_search(int nseg, int64_t x, KeyFn key) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (key(mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int seg_of_row(const SegDesc* sd, int nseg, int64_t row) {
  return seg_search(nseg, row, [&](int s) { return sd[s].q_off; });
}
__device__ __forceinline__ int seg_of_item(const SegDesc* sd, int nseg, int64_t item) {
  return seg_search(nseg, item, [&](int s) { return (int64_t)sd[s].item_off; });
}
__device__ __forceinline__ int seg_of_bigk(const SegDesc* sd, int nseg, int64_t x) {
  return seg_search(nseg, x, [&](int s) { return sd[s].bigk_off; });
}

}  // namespace knnag
