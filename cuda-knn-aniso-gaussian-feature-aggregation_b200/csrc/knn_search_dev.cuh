// Device helpers shared by the search kernels (knn_search.cu: the CUDA-core
// search and its plan; knn_search_tc.cu: the tensor-core filtered search):
// the sorted candidate list, the candidate queues, the seed thresholds and
// the tile lower bound.
#pragma once

#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {

// Insert (k, i) into the sorted list when k is below its top.  The list is
// ascending, so lt[s] = k < keys[s] is false up to the insertion point and
// true after it; every slot takes its left neighbour (lt[s-1]), the new
// entry (lt[s] only) or stays -- all comparisons are independent, so the
// insertion is a few instructions deep instead of a chain through the list.
// The entry that falls off the top is remembered when it was a real entry
// equal to the new top (a tie the exactness flags must see).
template <int L>
__device__ __forceinline__ void list_insert(float (&keys)[L], int (&vals)[L], float k, int i, float& tie_key) {
  bool lt[L];
#pragma unroll
  for (int s = 0; s < L; ++s) lt[s] = k < keys[s];
  const float out_k = keys[L - 1];
  const int out_i = vals[L - 1];
#pragma unroll
  for (int s = L - 1; s > 0; --s) {
    keys[s] = lt[s - 1] ? keys[s - 1] : (lt[s] ? k : keys[s]);
    vals[s] = lt[s - 1] ? vals[s - 1] : (lt[s] ? i : vals[s]);
  }
  keys[0] = lt[0] ? k : keys[0];
  vals[0] = lt[0] ? i : vals[0];
  if (lt[L - 1] && out_i >= 0 && out_k == keys[L - 1]) tie_key = fminf(tie_key, out_k);
}

// Queue slot of entry e of query (lane) j: rows are rotated by j so that
// appends (one query, consecutive entries) and drains (every lane its own
// query, the same entry) are both free of bank conflicts.
__device__ __forceinline__ int queue_slot(int j, int e) { return j * kQCap + ((e + j) & (kQCap - 1)); }

// Lane `lane` folds its query's n queued candidates into its list and
// refreshes its threshold; the caller resets the counts.
template <int L>
__device__ __forceinline__ void drain_queue(float (&keys)[L], int (&vals)[L], float& tie_key, float& tau, int n,
                                            const float* qk, const int* qv, int lane) {
  // the next entry is loaded while this one is folded in
  float k = n > 0 ? qk[queue_slot(lane, 0)] : 0.f;
  int i = n > 0 ? qv[queue_slot(lane, 0)] : -1;
  for (int e = 0; e < n; ++e) {
    const int s = queue_slot(lane, e + 1);
    const float kn = e + 1 < n ? qk[s] : 0.f;
    const int in = e + 1 < n ? qv[s] : -1;
    const float top = keys[L - 1];
    if (k < top) {
      list_insert<L>(keys, vals, k, i, tie_key);
    } else if (k == top) {
      tie_key = fminf(tie_key, k);
    }
    k = kn;
    i = in;
  }
  tau = fminf(tau, keys[L - 1]);
}

// Seed thresholds of a warp's NQ queries (NQ = 8, 16 or 32).  Any K+1
// distinct points bound a query's (K+1)-th smallest key from above by their
// own (K+1)-th smallest key, so keys above that can be dropped from the start
// instead of streaming through the list.  The points are a window of NS
// points of the sorted order around `my_seed` (held by lane j for query j:
// the middle of the query's cell, so the window is near it and the bound
// tight); the half-warp (the warp for NS = 64) of a query evaluates two
// points per lane and sorts the NS keys (bitonic, NaN as +inf), and the lane
// holding element K writes the bound into tab[j].w (tab[j] holds the query's
// x, y, z) for every valid query.  Nothing is written when P < NS.
template <int KMAX, int NQ>
__device__ __forceinline__ void seed_warp(float4* tab, int my_seed, bool valid, const float* pairs, int P, int K,
                                          int lane) {
  constexpr int NS = KMAX <= 16 ? 32 : 64;  // >= K + 1
  constexpr int LG = NS / 2;                // lanes per query
  constexpr int GPR = 32 / LG;              // queries per round
  constexpr int PPT = kTilePoints / 2;
  constexpr unsigned FULL = 0xffffffffu;
  static_assert((NQ / GPR) % 2 == 0, "two rounds per iteration");
  if (P >= NS) {
    const int gl = lane % LG;  // lane within the query's group
    const float2* pairs2 = reinterpret_cast<const float2*>(pairs);
    // two rounds per iteration: both windows' loads in flight together,
    // then the two sorts interleaved (NQ / GPR is even)
#pragma unroll 1
    for (int r = 0; r < NQ / GPR; r += 2) {
      int jj[2];
      bool qok[2];
      float2 pr[2][kRecLen];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        jj[u] = (r + u) * GPR + lane / LG;  // warp-local query of this group
        const int center = __shfl_sync(FULL, my_seed, jj[u]);
        qok[u] = __shfl_sync(FULL, valid, jj[u]);
        int a0 = center - NS / 2;
        a0 = (a0 < 0 ? 0 : (a0 > P - NS ? P - NS : a0)) & ~1;
        const int pos = a0 + 2 * gl;  // even, pos + 1 < P
        const float2* tp = pairs2 + (int64_t)(pos >> 7) * (PPT * kRecLen) + ((pos & (kTilePoints - 1)) >> 1);
#pragma unroll
        for (int f = 0; f < kRecLen; ++f) pr[u][f] = __ldg(tp + f * PPT);
      }
      float v0[2], v1[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const float4 qq = tab[jj[u]];
        const float2 s2 =
            key_pair(make_float2(qq.x, qq.x), make_float2(qq.y, qq.y), make_float2(qq.z, qq.z), pr[u]);
        v0[u] = s2.x == s2.x ? s2.x : INFINITY;
        v1[u] = s2.y == s2.y ? s2.y : INFINITY;
      }
      // element e = 2 * gl + h; ascending bitonic network over NS elements
#pragma unroll
      for (int kk = 2; kk <= NS; kk <<= 1) {
        const bool up = ((2 * gl) & kk) == 0;
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            if (j == 1) {
              const float lo = fminf(v0[u], v1[u]), hi = fmaxf(v0[u], v1[u]);
              v0[u] = up ? lo : hi;
              v1[u] = up ? hi : lo;
            } else {
              const float o0 = __shfl_xor_sync(FULL, v0[u], j >> 1), o1 = __shfl_xor_sync(FULL, v1[u], j >> 1);
              const bool take_min = (((2 * gl) & j) == 0) == up;
              v0[u] = take_min ? fminf(v0[u], o0) : fmaxf(v0[u], o0);
              v1[u] = take_min ? fminf(v1[u], o1) : fmaxf(v1[u], o1);
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (qok[u] && gl == (K >> 1)) tab[jj[u]].w = (K & 1) ? v1[u] : v0[u];
    }
  }
}

// One search work item: up to WPC * QPW queries of one batch element or
// segment, all against one cloud.  Pointers are offset to the group already.
struct SearchItem {
  const float* q;      // query rows (group-local index)
  const int* perm_q;   // sorted position -> group-local query index
  const float* rec;    // the cloud's records
  const float* pairs;  // the cloud's search tiles
  const float* tinfo;  // the cloud's tile infos (kTinfoFloats per tile)
  const float* f;      // the cloud's feature rows
  float* f_out;        // rows of the group's queries
  float* w_out;        // entries of the group's queries (K per query)
  float* dists;
  int64_t* idxs;
  int64_t row0;        // global query row of group-local query 0
  int* adj_count;      // the group's per-point entry counts (optional)
  const int* qseed;    // seed positions of the group's sorted queries (optional)
  const float* tau0;   // or their seed thresholds, from the plan kernel (optional)
  // or seeds from the query's cell: the scanned point counts of the
  // cloud's grid cells (global positions, cell 0 first), its box and grid
  const int* cell_start;
  const float* cbox;
  int cbits;
  int Q, P, K, ntile;
  int q0, q1;          // the item's queries: sorted positions [q0, q1), at most WPC * QPW
};

// Lower bound on the key of any query in box [bmin, bmax] against any point
// of a tile (its box ti[0..5], bound factor mu = ti[6]): mu * dist(box,
// tile box)^2, shrunk by 1e-5 for the rounding of this product; -inf when
// the tile has no bound (mu < 0).
__device__ __forceinline__ float tile_lower_bound(const float* ti, const float* bmin, const float* bmax) {
  const float mu = ti[6];
  if (!(mu >= 0.f)) return -INFINITY;
  float d2 = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float g = fmaxf(fmaxf(ti[c] - bmax[c], bmin[c] - ti[3 + c]), 0.f);
    d2 = __fmaf_rn(g, g, d2);
  }
  const float lb = mu * d2 * 0.99999f;
  return lb >= 0.f ? lb : 0.f;  // NaN: 0 (keys are >= 0 when mu >= 0)
}

}  // namespace knnag
