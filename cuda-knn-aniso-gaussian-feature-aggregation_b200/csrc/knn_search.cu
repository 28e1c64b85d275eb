// Forward path: point packing, the fused kNN search + aggregation kernel
// (FP32, K <= 32), and the exact MinK kernel that replays the reference's
// selection rules for flagged queries (and serves FP64 and K > 32).
//
// Replaces csrc/forward.cu:56-110 (kernel), csrc/forward.cu:286-338
// (launcher) and csrc/mink.cuh of the reference.
#include <math.h>

#include <algorithm>

#include "knn_common.cuh"
#include "knn_internal.h"
#include "knn_search_dev.cuh"

namespace knnag {

// ------------------------------------------------------------------ packing

// A record row (64 B / 128 B, 16-byte aligned) with 128-bit stores.
__device__ __forceinline__ void store_rec(float* dst, const float (&v)[kRecLen]) {
#pragma unroll
  for (int m = 0; m < kRecLen; m += 4)
    *reinterpret_cast<float4*>(dst + m) = make_float4(v[m], v[m + 1], v[m + 2], v[m + 3]);
}
__device__ __forceinline__ void store_rec(double* dst, const double (&v)[kRecLen]) {
#pragma unroll
  for (int m = 0; m < kRecLen; m += 2) *reinterpret_cast<double2*>(dst + m) = make_double2(v[m], v[m + 1]);
}

// One record from p, sigma, R (the shared body of the packing kernels).
template <typename T>
__device__ __forceinline__ void pack_one(const T* __restrict__ p, const T* __restrict__ sigma,
                                         const T* __restrict__ R, int64_t i, T* __restrict__ rec) {
  T v[kRecLen];
  v[kNPX] = -p[i * 3 + 0];
  v[kNPY] = -p[i * 3 + 1];
  v[kNPZ] = -p[i * 3 + 2];
#pragma unroll
  for (int m = 0; m < 9; ++m) v[kR00 + m] = R[i * 9 + m];
  v[kS0] = sigma[i * 3 + 0];
  v[kS1] = sigma[i * 3 + 1];
  v[kS2] = sigma[i * 3 + 2];
  v[kRecPad] = T(0);
  store_rec(rec + i * kRecLen, v);
}

// FP32 packing of the search path, grid (kBoundParts, B): CTA (c, b) packs
// chunk c of batch element b's points, writes the chunk's bounding box to
// parts (what the cell kernels reduce to the element's box), zeroes the
// chunk's adjacency counts (zero_rows, optional) and its share of the cell
// counts; CTA (0, 0) zeroes the call's status words.
__global__ void __launch_bounds__(256) pack_points_bounded_kernel(
    const float* __restrict__ p, const float* __restrict__ sigma, const float* __restrict__ R, int P,
    float* __restrict__ rec, float* __restrict__ parts, int* __restrict__ zero_words, int n_zero,
    int* __restrict__ zero_rows, int* __restrict__ zero_cells, int64_t n_cells) {
  __shared__ float red[6][8];
  const int c = blockIdx.x, b = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (c == 0 && b == 0 && tid < n_zero) zero_words[tid] = 0;
  const int64_t flat = ((int64_t)b * gridDim.x + c) * blockDim.x + tid;
  const int64_t nthreads = (int64_t)gridDim.x * gridDim.y * blockDim.x;
  for (int64_t i = flat; i < n_cells; i += nthreads) zero_cells[i] = 0;
  const int chunk = (P + kBoundParts - 1) / kBoundParts;
  const int i0 = min(P, c * chunk), i1 = min(P, i0 + chunk);
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int k = i0 + tid; k < i1; k += blockDim.x) {
    const int64_t i = (int64_t)b * P + k;
    pack_one<float>(p, sigma, R, i, rec);
    if (zero_rows) zero_rows[i] = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = p[i * 3 + a];
      mn[a] = fminf(mn[a], v);
      mx[a] = fmaxf(mx[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
      mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
    }
  if (lane == 0)
    for (int a = 0; a < 3; ++a) {
      red[a][warp] = mn[a];
      red[3 + a][warp] = mx[a];
    }
  __syncthreads();
  if (tid < 6) {
    float v = tid < 3 ? INFINITY : -INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = tid < 3 ? fminf(v, red[tid][w]) : fmaxf(v, red[tid][w]);
    parts[((int64_t)b * kBoundParts + c) * 8 + tid] = v;
  }
}

// rec[(b*P+i)*16 + field]: -p, R (row-major), sigma, pad.
// zero_rows (optional): one int per point zeroed too (the adjacency's
// per-point entry counts the forward accumulates).
template <typename T>
__global__ void pack_points_kernel(const T* __restrict__ p, const T* __restrict__ sigma,
                                   const T* __restrict__ R, int64_t n_points, T* __restrict__ rec,
                                   int* __restrict__ zero_words, int n_zero, int* __restrict__ zero_rows) {
  if (blockIdx.x == 0 && (int)threadIdx.x < n_zero) zero_words[threadIdx.x] = 0;  // the call's status words
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_points;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (zero_rows) zero_rows[i] = 0;
    pack_one<T>(p, sigma, R, i, rec);
  }
}

// ------------------------------------------------------------ exact MinK
//
// One CTA per query.  All threads compute the query's keys (same arithmetic
// as everywhere else) into shared memory, chunk by chunk; warp 0 then runs
// the reference's MinK selection over them in index order
// (csrc/mink.cuh:60-81):
//   fill:  the first K points take slots 0..K-1; the tracked maximum moves
//          only for the very first key or a strictly larger one;
//   full:  a point is taken only if strictly below the tracked maximum; it
//          overwrites the maximum's slot; the maximum is re-found by a strict
//          '>' scan that starts from the new key, i.e. it becomes the first
//          slot holding the largest key strictly above the new key, and stays
//          on the written slot when there is none;
//   sort:  bubble sort with a strict '<' swap (csrc/mink.cuh:99-112), which
//          without NaN keys is the stable sort by key.
// For K <= 32 slot s lives in lane s, so the re-scan is a warp max plus a
// ballot and the sort a stable rank; for K > 32, or when a kept key is NaN,
// lane 0 runs the rules sequentially on shared-memory slots.  A ballot
// skips keys that are not below the current maximum (it only falls, so they
// would be rejected anyway).

constexpr int kReplayThreads = 256;

template <typename T>
__host__ __device__ constexpr int replay_chunk() { return sizeof(T) == 4 ? 8192 : 4096; }

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T>
__device__ void bubble_sort_slots(T* sk, int* sv, int size) {
  for (int x = 0; x < size - 1; ++x)
    for (int y = 0; y < size - x - 1; ++y)
      if (sk[y + 1] < sk[y]) {
        const T tk = sk[y];
        const int tv = sv[y];
        sk[y] = sk[y + 1];
        sv[y] = sv[y + 1];
        sk[y + 1] = tk;
        sv[y + 1] = tv;
      }
}

template <typename T, int NTH>
__global__ void __launch_bounds__(NTH) mink_replay_kernel(ExactParams<T> a) {
  constexpr int CH = replay_chunk<T>();
  constexpr int HC = CH / 2;  // keys per chunk: two chunk buffers
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* skey = reinterpret_cast<T*>(smem_raw);
  T* slot_k = skey + CH;
  int* slot_v = reinterpret_cast<int*>(slot_k + a.K);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int F = a.F;
  const SegHeader* sh = static_cast<const SegHeader*>(a.segs);
  if (sh && *a.status) return;
  const int64_t n_items = a.use_list ? (int64_t)(*a.list_count)
                                     : (sh ? sh->bigk_q : (int64_t)a.B * a.Q);

  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    // bq: the query's global row; e0: its first entry; b: batch element
    // (uniform) -- records, features and sizes of its cloud
    int64_t bq, e0, b = 0;
    int K, P;
    const T* recb;
    const T* fb;
    if (sh) {
      const SegDesc* sd = seg_descs(a.segs);
      int s;
      if (a.use_list) {
        bq = a.list[item];
        if (bq < 0 || bq >= sh->total_q) {  // the search lists its own rows: never taken
          if (tid == 0) atomicOr(a.status, kStatusBadIndex);
          continue;
        }
        s = seg_of_row(sd, sh->nseg, bq);
      } else {
        s = seg_of_bigk(sd, sh->nseg, item);
        bq = sd[s].q_off + (item - sd[s].bigk_off);
      }
      const SegDesc g = sd[s];
      const CloudDesc c = cloud_descs(a.cs)[g.cloud];
      K = g.K;
      P = c.P;
      e0 = g.e_off + (bq - g.q_off) * K;
      recb = reinterpret_cast<const T*>(a.cs + reinterpret_cast<const CloudSetHeader*>(a.cs)->rec_off) +
             c.p_off * kRecLen;
      fb = a.f + c.p_off * F;
      if (K > a.K || K > P) continue;  // the host checked the table; never reached
    } else {
      bq = a.use_list ? (int64_t)a.list[item] : item;
      if (bq < 0 || bq >= (int64_t)a.B * a.Q) continue;  // the search lists its own rows: never taken
      b = bq / a.Q;
      K = a.K;
      P = a.P;
      e0 = bq * K;
      recb = a.rec + b * (int64_t)P * kRecLen;
      fb = a.f + b * (int64_t)P * F;
    }
    const bool in_lanes = K <= 32;
    const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];

    int size = 0, max_idx = 0, my_v = -1;
    T max_key = T(0), my_k = T(0);
    // Keys of chunk [c0, c0 + HC) into buf by threads first .. first + nth - 1
    // (four keys in flight per thread).
    auto fill = [&](int c0, T* buf, int first, int nth) {
      const int n = min(HC, P - c0);
      if (a.iso_p) {
        // squared Euclidean distance, accumulated as d = 0; d += c*c (csrc/forward.cu:32-36)
        const T* pb = a.iso_p + b * (int64_t)P * 3;
#pragma unroll 4
        for (int i = tid - first; i < n; i += nth) {
          const T* pp = pb + (int64_t)(c0 + i) * 3;
          const T x = qx - pp[0], y = qy - pp[1], z = qz - pp[2];
          buf[i] = fma_rn(z, z, fma_rn(y, y, mul_rn(x, x)));
        }
      } else {
#pragma unroll 4
        for (int i = tid - first; i < n; i += nth) buf[i] = key_rec<T>(qx, qy, qz, recb + (int64_t)(c0 + i) * kRecLen);
      }
    };
    // Two chunk buffers: while warp 0 runs MinK over chunk c in index order,
    // the other warps compute the keys of chunk c + 1.
    fill(0, skey, 0, NTH);
    __syncthreads();
    for (int c0 = 0, ci = 0; c0 < P; c0 += HC, ++ci) {
      const int n = min(HC, P - c0);
      const T* cur = skey + (ci & 1) * HC;
      if (warp != 0) {
        if (c0 + HC < P) fill(c0 + HC, skey + ((ci + 1) & 1) * HC, 32, NTH - 32);
      } else {
        // An accepted key kl (strictly below the max) at point index idx
        // replaces the max slot; the max is found again.
        auto accept = [&](T kl, int idx) {
          if (in_lanes) {
            if (lane == max_idx) {
              my_k = kl;
              my_v = idx;
            }
            const T v = (lane < K && my_k > kl) ? my_k : T(-INFINITY);
            const T m = warp_max(v);
            if (m > kl) {
              max_key = m;
              max_idx = __ffs(__ballot_sync(FULL, lane < K && v == m)) - 1;
            } else {
              max_key = kl;
            }
          } else {
            if (lane == 0) {
              slot_k[max_idx] = kl;
              slot_v[max_idx] = idx;
            }
            __syncwarp();
            max_key = kl;
            for (int s2 = 0; s2 < K; ++s2) {
              const T c = slot_k[s2];
              if (c > max_key) {
                max_key = c;
                max_idx = s2;
              }
            }
            __syncwarp();
          }
        };
        for (int base = 0; base < n;) {
          if (size >= K && base + 128 <= n) {
            // full list: 128 keys per step, lane l holding keys 4l .. 4l+3;
            // candidates in index order (lanes ascending, then t), each
            // checked against the max at its turn
            T k4[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) k4[t] = cur[base + 4 * lane + t];
            const bool any = k4[0] < max_key || k4[1] < max_key || k4[2] < max_key || k4[3] < max_key;
            unsigned cand = __ballot_sync(FULL, any);
            while (cand) {
              const int l = __ffs(cand) - 1;
              cand &= cand - 1;
#pragma unroll
              for (int t = 0; t < 4; ++t) {
                const T kl = __shfl_sync(FULL, k4[t], l);
                if (kl < max_key) accept(kl, c0 + base + 4 * l + t);
              }
            }
            base += 128;
            continue;
          }
          const int nvalid = min(32, n - base);
          const T key = lane < nvalid ? cur[base + lane] : T(0);
          int j = 0;
          while (j < nvalid && size < K) {  // fill phase (uniform across the warp)
            const T kj = __shfl_sync(FULL, key, j);
            if (in_lanes) {
              if (lane == size) {
                my_k = kj;
                my_v = c0 + base + j;
              }
            } else if (lane == 0) {
              slot_k[size] = kj;
              slot_v[size] = c0 + base + j;
            }
            if (size == 0 || kj > max_key) {
              max_key = kj;
              max_idx = size;
            }
            ++size;
            ++j;
          }
          __syncwarp();
          if (j < nvalid) {
            unsigned cand = __ballot_sync(FULL, lane >= j && lane < nvalid && key < max_key);
            while (cand) {
              const int l = __ffs(cand) - 1;
              cand &= cand - 1;
              const T kl = __shfl_sync(FULL, key, l);
              if (!(kl < max_key)) continue;
              accept(kl, c0 + base + l);
            }
          }
          base += 32;
        }
      }
      __syncthreads();
    }
    if (warp == 0) {
      if (in_lanes && !__any_sync(FULL, lane < K && my_k != my_k)) {
        int rank = 0;
        for (int t = 0; t < K; ++t) {
          const T kt = __shfl_sync(FULL, my_k, t);
          rank += (kt < my_k || (kt == my_k && t < lane)) ? 1 : 0;
        }
        if (lane < K) {
          slot_k[rank] = my_k;
          slot_v[rank] = my_v;
        }
      } else {
        if (in_lanes && lane < K) {
          slot_k[lane] = my_k;
          slot_v[lane] = my_v;
        }
        __syncwarp();
        if (lane == 0) bubble_sort_slots(slot_k, slot_v, size);
      }
    }
    __syncthreads();
    if (a.iso_p) {
      // isotropic weights w_k = exp(-(d_k * sigma[idx_k][0])) and their sum
      // in k order (csrc/forward.cu:43-52); keep w_k in slot_k
      const T* sg = a.iso_sigma + b * (int64_t)P * a.iso_stride;
      for (int k = tid; k < K; k += NTH) {
        const int64_t e = e0 + k;
        a.dists[e] = slot_k[k];
        a.idxs[e] = (int64_t)slot_v[k];
      }
      __syncthreads();
      for (int k = tid; k < K; k += NTH)
        slot_k[k] = weight_of(mul_rn(slot_k[k], sg[(int64_t)slot_v[k] * a.iso_stride]));
      __syncthreads();
      if (tid == 0) {
        T ws = T(0);
        for (int k = 0; k < K; ++k) ws = add_rn(ws, slot_k[k]);
        a.w_out[bq] = ws;
      }
    } else {
      for (int k = tid; k < K; k += NTH) {
        const int64_t e = e0 + k;
        a.dists[e] = slot_k[k];
        a.idxs[e] = (int64_t)slot_v[k];
        a.w_out[e] = weight_of(slot_k[k]);
        if (a.adj_count && (unsigned)slot_v[k] < (unsigned)P) atomicAdd(&a.adj_count[b * P + slot_v[k]], 1);
      }
      __syncthreads();
      for (int k = tid; k < K; k += NTH) slot_k[k] = weight_of(slot_k[k]);
      __syncthreads();
    }
    for (int c = tid; c < F; c += NTH) {
      T acc = T(0);
      for (int k = 0; k < K; ++k) acc = fma_rn(fb[(int64_t)slot_v[k] * F + c], slot_k[k], acc);
      a.f_out[bq * F + c] = acc;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------- fused FP32 search
//
// CTA = WPC warps (1, 2 or 4).  Each warp owns QPW queries (32, 16 or 8) --
// lane j < QPW keeps query j's sorted register list -- and all warps share
// the CTA's ring of point tiles (128 points, 8 KB, field-major: field f of
// pair m at float2 f * 64 + m), streamed into shared memory by
// one-dimensional bulk copies (TMA, no multicast), double-buffered on
// mbarriers.  Fewer queries per warp give more warps for small query sets.
//
// Keys are computed with lanes over POINTS: the warp's lanes form 32 / QPW
// slots of QPW lanes; in one pass a lane holds one point pair (16 float2
// registers, pair pass * QPW + lane % QPW of the tile) and every slot takes
// a different query the tile may matter to, broadcast from a shared table
// (x, y, z, threshold); one packed f32x2 evaluation gives the lane both of
// its points' keys, so a warp instruction covers 64 (query, point) pairs.
// Keys at or below the query's threshold are appended (ballot + popc
// positions) to the query's candidate queue in shared memory, and after
// every 64 points of a query each owner lane folds its queue into its
// list.  A query skips a tile whose lower bound against the query point
// exceeds its threshold.
//
// Selection.  Each list holds the K+1 smallest keys accepted so far in
// KMAX+1 slots whose lowest KMAX-K slots are -inf sentinels, so the
// (K+1)-th smallest real key is always the last slot; the threshold is that
// slot (stale values are still valid: lists only gain smaller keys).
//
// Exactness.  The result equals the reference's MinK selection whenever the
// K+1 smallest keys are pairwise distinct (then the top-K set and its order
// are unique) and no NaN key falls in MinK's fill phase (points 0..K-1).
// Every key that leaves a list or is not queued is either strictly above a
// threshold that is >= the (K+1)-th key, or equal to the threshold it was
// compared with; the smallest such "equal" key is tracked (tie_key).  A
// query is flagged for the exact replay kernel when its top-(K+1) holds
// equal keys or an empty slot, when tie_key <= its (K+1)-th key, or when a
// fill-phase key is NaN.

// The tile-ring mbarriers of a search CTA.
template <int WPC, int QPW>
__device__ __forceinline__ uint64_t* search_barriers(unsigned char* smem) {
  return reinterpret_cast<uint64_t*>(smem + search_bars_off(WPC, QPW));
}

// Search + aggregation of one work item.  The mbarriers are initialised by
// the kernel; uses[buf] counts the phases buffer buf has completed so far
// (a persistent CTA runs many items on the same barriers).  Returns false
// when a tile copy timed out (status flagged; the CTA must stop).
template <int KMAX, int WPC, int QPW>
__device__ __forceinline__ bool search_item(const SearchParams& a, const SearchItem& it, unsigned char* smem,
                                            int ntp_cap, uint32_t (&uses)[kTileBufs]) {
  constexpr int L = KMAX + 1;
  constexpr int NT = QPW * WPC;         // queries of the item
  constexpr int NTH = 32 * WPC;         // threads
  constexpr int H = 32 / QPW;           // lane slots per warp (queries evaluated at once)
  constexpr int PPT = kTilePoints / 2;  // pairs per tile
  constexpr int NPASS = PPT / QPW;      // passes per tile (QPW pairs each)
  constexpr unsigned FULL = 0xffffffffu;
  constexpr unsigned SLOT_MASK = QPW == 32 ? 0xffffffffu : ((1u << QPW) - 1u);
  static_assert(QPW == 32 || QPW == 16 || QPW == 8, "queries per warp");
  static_assert((size_t)NT * L * 12 + NT * 4 <= (size_t)WPC * search_warp_queue_bytes(QPW), "epilogue staging");

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool owner = lane < QPW;       // lane keeps query `lane` of the warp
  unsigned char* ring = smem;
  float* qk = reinterpret_cast<float*>(smem + search_queue_off() + (size_t)warp * search_warp_queue_bytes(QPW));
  int* qv = reinterpret_cast<int*>(qk + QPW * kQCap);
  float4* qtab = reinterpret_cast<float4*>(smem + search_qtab_off(WPC, QPW));  // [NT]
  float4* ctab = reinterpret_cast<float4*>(smem + search_ctab_off(WPC, QPW)) + warp * QPW;  // this warp's
  int* cidx = reinterpret_cast<int*>(smem + search_ctab_off(WPC, QPW) + (size_t)NT * 16) + warp * QPW;
  float* tring = reinterpret_cast<float*>(smem + search_tring_off(WPC, QPW));  // [kTileBufs][kTinfoFloats]
  int* qorig = reinterpret_cast<int*>(smem + search_misc_off(WPC, QPW));       // [NT] original query index (-1: none)
  float* qbox = reinterpret_cast<float*>(qorig + NT);                          // [WPC][6]
  uint64_t* full = search_barriers<WPC, QPW>(smem);
  int* cnt = reinterpret_cast<int*>(full + kTileBufs);               // warps done per buffer
  volatile int* s_final = reinterpret_cast<volatile int*>(cnt + kTileBufs);  // visit count once stopped
  volatile int* s_abort = s_final + 1;                               // a wait gave up
  // region C: per-tile lower bounds (sorted), visit order, visit counter
  const int NTP = search_tiles_pow2(it.ntile);
  float* lbk = reinterpret_cast<float*>(smem + search_smem_bytes(WPC, QPW));
  int* lbt = reinterpret_cast<int*>(lbk + ntp_cap);
  volatile int* s_nvisit = reinterpret_cast<volatile int*>(lbt + ntp_cap);
  volatile int* s_ncand = s_nvisit + 1;  // tiles in the visit order (the rest are never needed)
  // epilogue views of the queue region (after the tile loop)
  float* out_k = reinterpret_cast<float*>(smem + search_queue_off());
  int* out_i = reinterpret_cast<int*>(out_k + NT * L);
  float* out_w = reinterpret_cast<float*>(out_i + NT * L);
  int* out_f = reinterpret_cast<int*>(out_w + NT * L);

  // the item's queries split evenly over the warps (m <= QPW each: a split
  // item gives each warp fewer queries and so a shorter critical path)
  const int m = (it.q1 - it.q0 + WPC - 1) / WPC;
  const int lq = warp * QPW + lane;         // slot of this (owner) lane's query within the item
  const int sp = it.q0 + warp * m + lane;   // position in the spatial order
  bool valid = owner && lane < m && sp < it.q1;
  int qi = it.perm_q[valid ? sp : it.Q - 1];
  if ((unsigned)qi >= (unsigned)it.Q) {  // the query order is a permutation: never taken
    if (valid) atomicOr(a.status, kStatusBadIndex);
    qi = 0;
    valid = false;
  }
  const int K = it.K, P = it.P;
  const float qx = it.q[(int64_t)qi * 3 + 0], qy = it.q[(int64_t)qi * 3 + 1], qz = it.q[(int64_t)qi * 3 + 2];
  const float* recb = it.rec;
  if (owner) {
    qorig[lq] = valid ? qi : -1;
    qtab[lq] = make_float4(qx, qy, qz, valid ? INFINITY : -INFINITY);
  }

  // ---- seed thresholds (seed_warp): from the plan kernel when it ran,
  // else computed here from the query's cell
  const bool seeded = it.tau0 || it.qseed || it.cell_start;
  if (it.tau0) {  // computed by the plan kernel
    if (valid) qtab[lq].w = it.tau0[sp];
    __syncwarp();
  } else if (seeded) {
    int my_seed = 0;  // the middle of the query's cell in the sorted points
    if (valid) {
      if (it.qseed) {
        my_seed = it.qseed[sp];
      } else {
        const int c = (int)cell_of(qx, qy, qz, it.cbox, it.cbits);
        my_seed = ((it.cell_start[c] + it.cell_start[c + 1]) >> 1) - it.cell_start[0];
      }
    }
    __syncwarp();
    seed_warp<KMAX, QPW>(qtab + warp * QPW, my_seed, valid, it.pairs, P, K, lane);
    __syncwarp();
  }

  // MinK's fill phase stores points 0..K-1 whatever their key: a NaN there
  // changes the result in ways only the replay reproduces.  With those
  // records finite and at most 1e6 in magnitude, and the query too, no key
  // can overflow or be NaN (|key| < 1.2e32), so the keys are evaluated only
  // otherwise (lane i checks record i, K <= 32).
  bool fill_ok = true;
  if (lane < K) {
    float r[kRecLen];
    load_rec(recb + (int64_t)lane * kRecLen, r);
#pragma unroll
    for (int m = 0; m < kRecLen - 1; ++m) fill_ok = fill_ok && fabsf(r[m]) <= 1e6f;  // NaN fails
  }
  fill_ok = __all_sync(FULL, fill_ok) && fabsf(qx) <= 1e6f && fabsf(qy) <= 1e6f && fabsf(qz) <= 1e6f;
  bool nan_fill = false;
  if (owner && !fill_ok)
    for (int i = 0; i < K; ++i) {
      const float s = key_rec<float>(qx, qy, qz, recb + (int64_t)i * kRecLen);
      if (s != s) nan_fill = true;
    }

  // ---- box of this CTA's queries and the tile visit order
  {
    float bx[6] = {qx, qy, qz, qx, qy, qz};
    if (!valid) {
      bx[0] = bx[1] = bx[2] = INFINITY;
      bx[3] = bx[4] = bx[5] = -INFINITY;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bx[c] = fminf(bx[c], __shfl_xor_sync(FULL, bx[c], o));
        bx[3 + c] = fmaxf(bx[3 + c], __shfl_xor_sync(FULL, bx[3 + c], o));
      }
    }
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < 6; ++c) qbox[warp * 6 + c] = bx[c];
  }
  __syncthreads();
  float bmin[3], bmax[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    bmin[c] = qbox[c];
    bmax[c] = qbox[3 + c];
#pragma unroll
    for (int w = 1; w < WPC; ++w) {
      bmin[c] = fminf(bmin[c], qbox[w * 6 + c]);
      bmax[c] = fmaxf(bmax[c], qbox[w * 6 + 3 + c]);
    }
  }
  const float* tinfo_b = it.tinfo;
  // Seeded queries bound the tiles worth visiting: a tile whose bound
  // against the CTA's box exceeds every query's seed holds no point below
  // any threshold the search will ever use.  Only the tiles at or below the
  // largest seed are sorted (all of them without seeds).
  float tmax0 = INFINITY;
  if (seeded) {
    tmax0 = -INFINITY;
    for (int i = lane; i < NT; i += 32) tmax0 = fmaxf(tmax0, qtab[i].w);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tmax0 = fmaxf(tmax0, __shfl_xor_sync(FULL, tmax0, o));
  }
  // (bound, tile) ascending, ties by tile, in registers across warp 0's
  // lanes (shuffle bitonic network); invalid entries carry +inf.
  auto warp_sort_tiles = [&](float& lb, int& ti) {
#pragma unroll
    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
      for (int j = kk >> 1; j > 0; j >>= 1) {
        const float ok = __shfl_xor_sync(FULL, lb, j);
        const int oi = __shfl_xor_sync(FULL, ti, j);
        const bool up = (lane & kk) == 0;
        const bool lower = (lane & j) == 0;
        const bool other_less = ok < lb || (ok == lb && oi < ti);
        if (lower == up ? other_less : !other_less) {
          lb = ok;
          ti = oi;
        }
      }
    }
  };
  if (NTP <= 32) {
    // Up to 32 tiles: warp 0 computes the bounds and sorts them in registers.
    if (warp == 0) {
      float lb = INFINITY;
      int ti = lane;
      bool keep = false;
      if (lane < it.ntile) {
        lb = tile_lower_bound(tinfo_b + lane * kTinfoFloats, bmin, bmax);
        keep = !(lb > tmax0);
        lb = keep ? fminf(lb, 3.4e38f) : INFINITY;  // kept tiles sort before the rest
      }
      const int nkeep = __popc(__ballot_sync(FULL, keep));
      warp_sort_tiles(lb, ti);
      if (lane < NTP) {
        lbk[lane] = lb;
        lbt[lane] = ti;
      }
      if (lane == 0) *s_ncand = nkeep;
    }
    __syncthreads();
  } else {
    // Compact the kept tiles (in any order), then sort them: in warp 0's
    // registers when at most 32, else in shared memory over the next power
    // of two (padding +inf).
    if (tid == 0) *s_ncand = 0;
    __syncthreads();
    for (int t = tid; t < it.ntile; t += NTH) {
      const float lb = tile_lower_bound(tinfo_b + (int64_t)t * kTinfoFloats, bmin, bmax);
      if (!(lb > tmax0)) {
        const int pos = atomicAdd(const_cast<int*>(s_ncand), 1);
        lbk[pos] = fminf(lb, 3.4e38f);
        lbt[pos] = t;
      }
    }
    __syncthreads();
    const int nkeep = *s_ncand;
    if (nkeep <= 32) {
      if (warp == 0) {
        float lb = lane < nkeep ? lbk[lane] : INFINITY;
        int ti = lane < nkeep ? lbt[lane] : 0x7fffffff;
        warp_sort_tiles(lb, ti);
        if (lane < nkeep) {
          lbk[lane] = lb;
          lbt[lane] = ti;
        }
      }
      __syncthreads();
    } else {
      const int ns = search_tiles_pow2(nkeep);  // <= NTP
      for (int t = nkeep + tid; t < ns; t += NTH) {
        lbk[t] = INFINITY;
        lbt[t] = 0x7fffffff;
      }
      __syncthreads();
      for (int kk = 2; kk <= ns; kk <<= 1) {  // bitonic sort of (bound, tile) ascending
        for (int j = kk >> 1; j > 0; j >>= 1) {
          for (int i = tid; i < ns; i += NTH) {
            const int ixj = i ^ j;
            if (ixj > i) {
              const bool up = (i & kk) == 0;
              const float ki = lbk[i], kj = lbk[ixj];
              const int ti = lbt[i], tj = lbt[ixj];
              if ((ki > kj || (ki == kj && ti > tj)) == up) {
                lbk[i] = kj;
                lbk[ixj] = ki;
                lbt[i] = tj;
                lbt[ixj] = ti;
              }
            }
          }
          __syncthreads();
        }
      }
    }
  }

  float keys[L];
  int vals[L];
#pragma unroll
  for (int s = 0; s < L; ++s) {
    keys[s] = (s < KMAX - K) ? -INFINITY : INFINITY;
    vals[s] = -1;
  }
  float tau = owner ? qtab[lq].w : -INFINITY, tie_key = INFINITY;  // the seed, +inf or -inf (no query)
  int my_cnt = 0;  // queued candidates of this lane's query
  const float qpt[3] = {qx, qy, qz};

  const int ntile = it.ntile;
  const float* pairs_b = it.pairs;
  // visit position v reads tile lbt[v] into buffer v % kTileBufs
  auto issue = [&](int v) {
    const int buf = v % kTileBufs;
    mbar_arrive_expect_tx(&full[buf], (uint32_t)kSearchTileBytes + kTinfoBytes);
    if (v == a.stall_visit) return;  // test hook: this phase never completes
    bulk_copy_g2s(ring + buf * kSearchTileBytes, pairs_b + (int64_t)lbt[v] * PPT * kPairFloats,
                  (uint32_t)kSearchTileBytes, &full[buf]);
    bulk_copy_g2s(tring + buf * kTinfoFloats, tinfo_b + (int64_t)lbt[v] * kTinfoFloats, kTinfoBytes, &full[buf]);
  };
  // Issue position v unless its bound exceeds every threshold (the order is
  // ascending, so nothing after it is needed either).  Decisions are made
  // one visit at a time, in order (see below), so *s_nvisit == v here.
  auto decide = [&](int v, float tmax) {
    if (v >= *s_ncand || *s_nvisit != v) return false;
    if ((unsigned)lbt[v] >= (unsigned)ntile) {  // real tiles sort first: never taken
      atomicOr(a.status, kStatusBadIndex);
      return false;
    }
    if (lbk[v] > tmax) return false;
    *s_nvisit = v + 1;
    return true;
  };
  // No visit v: record the count and complete its buffer's next phase with
  // a plain arrive, so the warps waiting for visit v wake up and stop.
  auto stop = [&](int v) {
    *s_final = v;
    __threadfence_block();
    mbar_arrive(&full[v % kTileBufs]);
  };
  if (tid == 0) {
    *s_nvisit = 0;
    *s_final = 0x7fffffff;
    *s_abort = 0;
    for (int b = 0; b < kTileBufs; ++b) cnt[b] = 0;
    fence_proxy_async_smem();  // the ring was last written by generic stores
    for (int v = 0; v < kTileBufs; ++v) {
      if (decide(v, INFINITY)) {
        issue(v);
      } else {
        stop(v);
        break;
      }
    }
  }
  __syncthreads();

  // Tile loop without CTA barriers.  Visit t sits in buffer t % kTileBufs;
  // each warp waits for its copy, evaluates the tile for its queries that
  // need it, publishes its thresholds and counts itself out of the tile.
  // The warp that counts out last knows every warp is done with the
  // buffer: it re-arms the counter and decides (and issues) visit
  // t + kTileBufs into the same buffer.  A warp does that duty before it
  // starts its next tile, so the decision for t + kTileBufs - 1 is complete
  // before any warp can be last for tile t: decisions stay in order.
  int t = 0;
  for (;; ++t) {
    const int buf = t % kTileBufs;
    const bool ok = mbar_wait_bounded(&full[buf], (uses[buf] + t / kTileBufs) & 1, a.wait_spins);
    if (!ok) {
      if (lane == 0) {
        atomicOr(a.status, kStatusWaitTimeout);
        *s_abort = 1;
      }
      break;
    }
    if (*s_abort || t >= *s_final) break;
    const float2* tile = reinterpret_cast<const float2*>(ring + buf * kSearchTileBytes);
    // queries of this warp the tile may matter to: bound against the query
    // point itself not above its threshold
    const float* tinf = tring + buf * kTinfoFloats;  // the tile's box, then its sub-boxes
    const float lbq = tile_lower_bound(tinf, qpt, qpt);
    const unsigned need = __ballot_sync(FULL, valid && !(lbq > tau));
    if (need) {
      constexpr int SPP = QPW >= 16 ? QPW / 16 : 1;  // sub-boxes a pass covers (2 QPW points)
      const int slot = lane / QPW;
      const unsigned my_mask = SLOT_MASK << (slot * QPW);
      const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll 1
      for (int pass = 0; pass < NPASS; ++pass) {
        // The queries this pass matters to: the tile's, less those whose
        // bound against the pass's sub-box exceeds their threshold,
        // compacted in lane order (round r slot h takes entry r * H + h).
        // Owner lanes publish their entry and keep its rank (refreshed
        // thresholds go there too).
        const int sb0 = (2 * pass * QPW) / 32;
        float lbp = INFINITY;
#pragma unroll
        for (int u = 0; u < SPP; ++u) lbp = fminf(lbp, tile_lower_bound(tinf + 8 * (1 + sb0 + u), qpt, qpt));
        const unsigned need_p = __ballot_sync(FULL, ((need >> lane) & 1u) && !(lbp > tau));
        const int n_need = __popc(need_p);
        const int my_rank = ((need_p >> lane) & 1u) ? __popc(need_p & lt_mask) : -1;
        if (need_p) {
          const int R = (n_need + H - 1) / H;  // rounds of this pass
          const int my_round = my_rank >= 0 ? my_rank / H : -1;
          const unsigned my_slot_mask = SLOT_MASK << ((my_rank >= 0 ? my_rank % H : 0) * QPW);
          __syncwarp();  // the previous pass's readers are done with the table
          if (my_rank >= 0) {
            ctab[my_rank] = make_float4(qx, qy, qz, tau);
            cidx[my_rank] = lane;
          }
          __syncwarp();
          float2 pr[kRecLen];
          const int pidx = pass * QPW + (lane & (QPW - 1));
#pragma unroll
          for (int f = 0; f < kRecLen; ++f) pr[f] = tile[f * PPT + pidx];
          const int i0 = __float_as_int(pr[kRecPad].x), i1 = __float_as_int(pr[kRecPad].y);
#pragma unroll 1
          for (int r0 = 0; r0 < R; r0 += 2) {
            // two rounds per iteration (independent key evaluations in flight)
            int jr[2];
            float4 qr[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int e = (r0 + u) * H + slot;
              jr[u] = e < n_need ? cidx[e] : -1;
              qr[u] = ctab[e < n_need ? e : 0];
            }
            float2 sr[2];
#pragma unroll
            for (int u = 0; u < 2; ++u)
              sr[u] = key_pair(make_float2(qr[u].x, qr[u].x), make_float2(qr[u].y, qr[u].y),
                               make_float2(qr[u].z, qr[u].z), pr);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              if (u == 1 && r0 + 1 >= R) break;  // warp-uniform: no round 1
              const int j = jr[u];
              const float2 s2 = sr[u];
              const bool c0 = j >= 0 && s2.x <= qr[u].w, c1 = j >= 0 && s2.y <= qr[u].w;
              const unsigned b0 = __ballot_sync(FULL, c0), b1 = __ballot_sync(FULL, c1);
              if (b0 | b1) {
                const int n = __popc(b0 & my_mask) + __popc(b1 & my_mask);
                int c = __shfl_sync(FULL, my_cnt, j >= 0 ? j : 0);
                if (__any_sync(FULL, j >= 0 && c + n > kQCap)) {  // a queue would overflow: fold every queue first
                  __syncwarp();
                  drain_queue<L>(keys, vals, tie_key, tau, my_cnt, qk, qv, lane);
                  my_cnt = 0;
                  if (owner) qtab[lq].w = tau;
                  if (my_rank >= 0) ctab[my_rank].w = tau;
                  __syncwarp();
                  c = 0;
                }
                if (c0) {
                  const int e = queue_slot(j, c + __popc(b0 & my_mask & lt_mask));
                  qk[e] = s2.x;
                  qv[e] = i0;
                }
                if (c1) {
                  const int e = queue_slot(j, c + __popc(b0 & my_mask) + __popc(b1 & my_mask & lt_mask));
                  qk[e] = s2.y;
                  qv[e] = i1;
                }
                if (my_round == r0 + u) my_cnt += __popc(b0 & my_slot_mask) + __popc(b1 & my_slot_mask);
              }
            }
          }
        }
        if ((pass + 1) % H == 0) {  // every query met at most 64 more points since the last fold
          __syncwarp();
          drain_queue<L>(keys, vals, tie_key, tau, my_cnt, qk, qv, lane);
          my_cnt = 0;
          if (owner) qtab[lq].w = tau;
          if (my_rank >= 0) ctab[my_rank].w = tau;
          __syncwarp();
        }
      }
    }
    // count this warp out of the tile (release: its reads of the buffer and
    // its threshold writes come first)
    __syncwarp();
    int last = 0;
    if (lane == 0) {
      __threadfence_block();
      last = atomicAdd(&cnt[buf], 1) == WPC - 1;
      if (last) __threadfence_block();
    }
    last = __shfl_sync(FULL, last, 0);
    if (last) {
      // every warp is done with this buffer: re-arm its counter, then decide
      // visit t + kTileBufs unless a stop was made; a tile is needed while
      // its bound is below some query's threshold
      float tmax = -INFINITY;
      for (int i = lane; i < NT; i += 32) tmax = fmaxf(tmax, qtab[i].w);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tmax = fmaxf(tmax, __shfl_xor_sync(FULL, tmax, o));
      if (lane == 0) {
        cnt[buf] = 0;
        if (*s_final == 0x7fffffff && !*s_abort) {
          if (decide(t + kTileBufs, tmax)) {
            fence_proxy_async_smem();
            issue(t + kTileBufs);
          } else {
            stop(t + kTileBufs);
          }
        }
      }
    }
  }
  // Every warp has left the loop once all meet here; no copy is in flight
  // then (each issued visit was waited for by every warp), unless a wait
  // gave up.
  __syncthreads();
  if (*s_abort) {
    if (tid == 0) {
      // best effort: let the copies of the last issued visits land
      for (int v = *s_nvisit - kTileBufs; v < *s_nvisit; ++v)
        if (v >= 0) mbar_wait_bounded(&full[v % kTileBufs], (uses[v % kTileBufs] + v / kTileBufs) & 1, a.wait_spins);
    }
    return false;
  }
  {
    const int n = t + 1;  // phases waited on: visits 0..t (t = the stop visit)
#pragma unroll
    for (int b = 0; b < kTileBufs; ++b) uses[b] += n > b ? (n - b + kTileBufs - 1) / kTileBufs : 0;
  }

  // ---- flags and staging; the queue region is free (every drain ended
  // before the last barrier)
  if (owner) {
#pragma unroll
    for (int s = 0; s < L; ++s) {
      const int j = s - (KMAX - K);
      if (j >= 0) {
        out_k[lq * L + j] = keys[s];
        out_i[lq * L + j] = vals[s];
      }
    }

    const int nneed = (P > K) ? K + 1 : K;
    bool fl = nan_fill, bad = false;
    for (int j = 0; j < nneed; ++j) {
      const int idx = out_i[lq * L + j];
      if (idx < 0) fl = true;
      if (idx >= P) bad = true;  // tiles carry indices of their own cloud: never taken
    }
    if (bad && valid) atomicOr(a.status, kStatusBadIndex);
    for (int j = 0; j + 1 < nneed; ++j)
      if (out_k[lq * L + j] == out_k[lq * L + j + 1]) fl = true;
    const float m = (P > K) ? out_k[lq * L + K] : INFINITY;
    if (tie_key <= m) fl = true;
    for (int j = 0; j < K; ++j) out_w[lq * L + j] = weight_of(out_k[lq * L + j]);
    out_f[lq] = (fl || bad || !valid) ? 1 : 0;
    if (valid && fl && !bad) {
      const int pos = atomicAdd(a.flag_count, 1);
      a.flag_list[pos] = (int)(it.row0 + qi);
    }
  }
  __syncthreads();

  // ---- epilogue: dists / idxs / w_out, then f_out = sum_k w_k f[idx_k]
  // accumulated in k order with fma, 128-bit gathers of f rows.  Rows go to
  // the queries' original positions.
  for (int x = tid; x < NT * K; x += NTH) {
    const int l = x / K, k = x - l * K;
    if (out_f[l]) continue;
    const int64_t e = (int64_t)qorig[l] * K + k;
    const int idx = out_i[l * L + k];
    it.dists[e] = out_k[l * L + k];
    it.idxs[e] = (int64_t)idx;
    it.w_out[e] = out_w[l * L + k];
    if (it.adj_count) atomicAdd(&it.adj_count[idx], 1);  // idx is in [0, P): unflagged
  }
  const int F = a.F;
  const float* fb = it.f;
  if (a.vec4) {
    const int C4 = F >> 2;
    for (int x = tid; x < NT * C4; x += NTH) {
      const int l = x / C4, c = x - l * C4;
      if (out_f[l]) continue;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      // sixteen rows in flight, summed in k order
      constexpr int RB = 16;
      for (int k0 = 0; k0 < K; k0 += RB) {
        float4 v[RB];
        float w[RB];
#pragma unroll
        for (int j = 0; j < RB; ++j) {
          const bool in = k0 + j < K;
          const int idx = in ? out_i[l * L + k0 + j] : 0;
          w[j] = in ? out_w[l * L + k0 + j] : 0.f;
          v[j] = in ? __ldg(reinterpret_cast<const float4*>(fb + (int64_t)idx * F) + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < RB; ++j) {
          if (k0 + j < K) {
            acc.x = __fmaf_rn(v[j].x, w[j], acc.x);
            acc.y = __fmaf_rn(v[j].y, w[j], acc.y);
            acc.z = __fmaf_rn(v[j].z, w[j], acc.z);
            acc.w = __fmaf_rn(v[j].w, w[j], acc.w);
          }
        }
      }
      reinterpret_cast<float4*>(it.f_out + (int64_t)qorig[l] * F)[c] = acc;
    }
  } else {
    for (int x = tid; x < NT * F; x += NTH) {
      const int l = x / F, c = x - l * F;
      if (out_f[l]) continue;
      float acc = 0.f;
      for (int k = 0; k < K; ++k)
        acc = __fmaf_rn(__ldg(fb + (int64_t)out_i[l * L + k] * F + c), out_w[l * L + k], acc);
      it.f_out[(int64_t)qorig[l] * F + c] = acc;
    }
  }
  return true;
}

template <int KMAX, int WPC, int QPW>
__global__ void __launch_bounds__(32 * WPC) search_f32_kernel(SearchParams a) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = search_barriers<WPC, QPW>(smem);
  if (threadIdx.x == 0) {
    for (int b = 0; b < kTileBufs; ++b) mbar_init(&full[b], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // the plan kernel's item (batch element, sorted query range), else block
  // (blockIdx.x, blockIdx.y) of WPC * QPW queries
  int64_t b = blockIdx.y;
  int q0 = blockIdx.x * (WPC * QPW), q1 = min(q0 + WPC * QPW, a.Q);
  if (a.items) {
    const int4 itm = a.items[blockIdx.x];
    b = itm.x;
    q0 = itm.y;
    q1 = itm.z;
  }
  SearchItem it;
  it.q = a.q + b * a.Q * 3;
  it.perm_q = a.perm_q + b * a.Q;
  it.rec = a.rec + b * a.P * kRecLen;
  it.pairs = a.pairs + b * (a.P_pad / 2) * kPairFloats;
  it.tinfo = a.tinfo + b * a.ntile * kTinfoFloats;
  it.f = a.f + b * a.P * a.F;
  it.f_out = a.f_out + b * a.Q * a.F;
  it.w_out = a.w_out + b * a.Q * a.K;
  it.dists = a.dists + b * a.Q * a.K;
  it.idxs = a.idxs + b * a.Q * a.K;
  it.row0 = b * a.Q;
  it.adj_count = a.adj_count ? a.adj_count + b * a.P : nullptr;
  it.qseed = a.qseed ? a.qseed + b * a.Q : nullptr;
  it.cell_start = nullptr;
  it.cbox = nullptr;
  it.cbits = 0;
  it.Q = a.Q;
  it.P = a.P;
  it.K = a.K;
  it.ntile = a.ntile;
  it.q0 = q0;
  it.q1 = q1;
  it.tau0 = a.items ? a.tau0 + b * a.Q : nullptr;
  uint32_t uses[kTileBufs] = {};
  search_item<KMAX, WPC, QPW>(a, it, smem, search_tiles_pow2(a.ntile), uses);
}

// ------------------------------------------------------------ search plan
//
// search_plan_kernel, one CTA per block of qpc sorted queries (grid (nb, B),
// 16 queries per warp): the seed thresholds of the block's queries
// (seed_warp) into tau0, and the block's estimate -- the number of tiles
// whose bound against the block's query box is at most its largest seed,
// the tiles its search may visit -- into plan_est.
// search_items_kernel, one CTA of 1024 threads, turns the estimates into the
// search's CTA items (batch element, query range): blocks ordered by
// estimate, heaviest first, in kPlanGroups groups of about equal population
// (block order inside a group), so the heaviest blocks start in the first
// waves and the light ones fill the last.  The plan runs only when the
// blocks take more than one wave: in one wave every block starts at once and
// the order changes nothing (splitting the heaviest blocks over the spare
// slots of a wave was measured, and gained less than the plan cost).
// Items only decide which CTA runs which queries: results do not change.
constexpr int kPlanBins = 1024;
constexpr int kPlanGroups = 8;
constexpr int kPlanQPW = 16;              // queries per warp of the plan kernel
constexpr int kPlanItemsThreads = 1024;
constexpr int kPlanMaxBlocks = 32768;     // estimates staged in shared memory (128 KB)

// Exclusive scan of one int per thread over the CTA; *total gets the sum.
// wsum: 33 ints of shared memory.  Every thread of the CTA must call it.
__device__ __forceinline__ int cta_scan_excl(int v, int* wsum, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < nw ? wsum[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nw) wsum[lane] = wi - w;
    if (lane == 31) wsum[32] = wi;
  }
  __syncthreads();
  const int r = wsum[warp] + incl - v;
  *total = wsum[32];
  __syncthreads();  // wsum is reused by the next call
  return r;
}

__device__ __forceinline__ int4 plan_item(int bt, int nb, int qpc, int Q) {
  const int b = bt / nb, blk = bt - b * nb;
  const int q0 = blk * qpc;
  return make_int4(b, q0, min(q0 + qpc, Q), 0);
}

template <int KMAX>
__global__ void __launch_bounds__(256) search_plan_kernel(SearchParams a, int qpc, int nb) {
  constexpr int NQ = kPlanQPW;
  __shared__ float4 tab[256 / 32 * NQ];
  __shared__ float red[8][8];
  __shared__ int wsum[33];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const int b = blockIdx.y, blk = blockIdx.x;
  const int q0 = blk * qpc, q1 = min(q0 + qpc, a.Q);
  const int sp = q0 + warp * NQ + lane;
  const bool valid = lane < NQ && sp < q1;
  const int64_t qrow = (int64_t)b * a.Q;
  int qi = valid ? a.perm_q[qrow + sp] : 0;
  if ((unsigned)qi >= (unsigned)a.Q) qi = 0;  // the search flags a bad permutation
  const float* qb = a.q + qrow * 3;
  const float x = qb[(int64_t)qi * 3 + 0], y = qb[(int64_t)qi * 3 + 1], z = qb[(int64_t)qi * 3 + 2];
  if (lane < NQ) tab[warp * NQ + lane] = make_float4(x, y, z, INFINITY);
  const int my_seed = valid ? a.qseed[qrow + sp] : 0;
  __syncwarp();
  seed_warp<KMAX, NQ>(tab + warp * NQ, my_seed, valid, a.pairs + (int64_t)b * (a.P_pad / 2) * kPairFloats, a.P,
                      a.K, lane);
  __syncwarp();
  float t0 = -INFINITY;
  if (valid) {
    t0 = tab[warp * NQ + lane].w;
    a.tau0[qrow + sp] = t0;
  }
  // the block's query box and largest seed
  float v[7] = {valid ? x : INFINITY,  valid ? y : INFINITY,  valid ? z : INFINITY, valid ? x : -INFINITY,
                valid ? y : -INFINITY, valid ? z : -INFINITY, t0};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = fminf(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
#pragma unroll
    for (int c = 3; c < 7; ++c) v[c] = fmaxf(v[c], __shfl_xor_sync(0xffffffffu, v[c], o));
  }
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < 7; ++c) red[warp][c] = v[c];
  __syncthreads();
  float bmin[3], bmax[3], tmax0 = -INFINITY;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    bmin[c] = INFINITY;
    bmax[c] = -INFINITY;
  }
  for (int w = 0; w < nw; ++w) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      bmin[c] = fminf(bmin[c], red[w][c]);
      bmax[c] = fmaxf(bmax[c], red[w][3 + c]);
    }
    tmax0 = fmaxf(tmax0, red[w][6]);
  }
  // the tiles the block's search may visit
  const float* tinfo_b = a.tinfo + (int64_t)b * a.ntile * kTinfoFloats;
  int c = 0;
  for (int t = tid; t < a.ntile; t += blockDim.x)
    c += tile_lower_bound(tinfo_b + (int64_t)t * kTinfoFloats, bmin, bmax) > tmax0 ? 0 : 1;
  int est;
  cta_scan_excl(c, wsum, &est);
  if (tid == 0) a.plan_est[(int64_t)b * nb + blk] = est;
}

// The item table from the estimates of nbt = B * nb blocks (one CTA of
// kPlanItemsThreads threads; dynamic shared memory: nbt ints).
__global__ void __launch_bounds__(kPlanItemsThreads) search_items_kernel(SearchParams a, int nb, int qpc) {
  extern __shared__ int est[];  // [nbt]
  __shared__ int hist[kPlanBins];
  __shared__ int wsum[33];
  __shared__ int misc[2 * kPlanGroups];
  const int tid = threadIdx.x, nth = blockDim.x;
  const int nbt = a.B * nb;
  const int nbins = a.ntile + 1 < kPlanBins ? a.ntile + 1 : kPlanBins;  // estimates are in [0, ntile]
  for (int i = tid; i < nbt; i += nth) {
    const int e = a.plan_est[i];
    est[i] = e < nbins - 1 ? e : nbins - 1;  // the bin
  }
  for (int i = tid; i < kPlanBins; i += nth) hist[i] = 0;
  if (tid < 2 * kPlanGroups) misc[tid] = 0;
  __syncthreads();
  for (int i = tid; i < nbt; i += nth) atomicAdd(&hist[est[i]], 1);
  __syncthreads();
  // blocks in bins above bin t (heaviest first): one bin per thread
  const int t = nbins - 1 - tid;  // thread tid holds bin t (tid < nbins)
  const int h = tid < nbins ? hist[t] : 0;
  int tot;
  const int above = cta_scan_excl(h, wsum, &tot);
  const int chunk = (nbt + nth - 1) / nth;  // thread tid takes blocks [i0, i1) in order
  const int i0 = min(nbt, tid * chunk), i1 = min(nbt, i0 + chunk);
  // group of each bin (heaviest bins first), each group's size and first item
  __syncthreads();  // every thread read its bin's count
  if (tid < nbins) {
    const int g = min(kPlanGroups - 1, (int)((int64_t)above * kPlanGroups / nbt));
    hist[t] = g;
    atomicAdd(&misc[g], h);
  }
  __syncthreads();
  if (tid == 0) {
    int o = 0;
    for (int g = 0; g < kPlanGroups; ++g) {
      misc[kPlanGroups + g] = o;
      o += misc[g];
    }
  }
  __syncthreads();
  int cnt[kPlanGroups], base[kPlanGroups];
#pragma unroll
  for (int g = 0; g < kPlanGroups; ++g) cnt[g] = 0;
  for (int i = i0; i < i1; ++i) {
    const int g = hist[est[i]];
#pragma unroll
    for (int u = 0; u < kPlanGroups; ++u) cnt[u] += g == u ? 1 : 0;
  }
#pragma unroll
  for (int g = 0; g < kPlanGroups; ++g) base[g] = misc[kPlanGroups + g] + cta_scan_excl(cnt[g], wsum, &tot);
  for (int i = i0; i < i1; ++i) {
    const int g = hist[est[i]];
    int p = 0;
#pragma unroll
    for (int u = 0; u < kPlanGroups; ++u)
      if (g == u) p = base[u]++;
    a.items[p] = plan_item(i, nb, qpc, a.Q);
  }
}

// Ragged search: a persistent CTA takes work items in order from a counter
// until the segment table's items run out.  Item i belongs to the last
// segment whose item_off <= i; its queries are that segment's sorted
// positions [(i - item_off) * WPC * QPW, ...).  Each item runs with the
// register list of its own segment's K (8, 16 or 32 slots + 1), up to the
// launch's KMAX.
template <int KMAX, int WPC, int QPW>
__global__ void __launch_bounds__(32 * WPC) search_ragged_kernel(SearchParams a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_item;
  if (*a.status) return;  // the table failed validation
  uint64_t* full = search_barriers<WPC, QPW>(smem);
  if (threadIdx.x == 0) {
    for (int b = 0; b < kTileBufs; ++b) mbar_init(&full[b], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const SegHeader* sh = static_cast<const SegHeader*>(a.segs);
  const SegDesc* sd = seg_descs(a.segs);
  const CloudSetHeader* ch = reinterpret_cast<const CloudSetHeader*>(a.cs);
  const CloudDesc* cd = cloud_descs(a.cs);
  const float* crec = reinterpret_cast<const float*>(a.cs + ch->rec_off);
  const float* cpairs = reinterpret_cast<const float*>(a.cs + ch->pairs_off);
  const float* ctinfo = reinterpret_cast<const float*>(a.cs + ch->tinfo_off);
  const float* cbnd = reinterpret_cast<const float*>(a.cs + ch->bnd_off);
  const int* ccell = reinterpret_cast<const int*>(a.cs + ch->celloff_off);
  const int nseg = sh->nseg, n_items = sh->n_items;
  const int ntp_cap = search_tiles_pow2(a.ntile);
  constexpr int QPC = WPC * QPW;
  uint32_t uses[kTileBufs] = {};
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.item_counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= n_items) break;
    if (item < 0) {  // the counter starts at 0 and only grows: never taken
      if (threadIdx.x == 0) atomicOr(a.status, kStatusBadIndex);
      break;
    }
    const SegDesc g = sd[seg_of_item(sd, nseg, item)];
    const CloudDesc c = cd[g.cloud];
    if (g.K < 1 || g.K > KMAX || g.K > c.P || c.ntile > a.ntile || sh->qpc != QPC) {
      if (threadIdx.x == 0) atomicOr(a.status, kStatusBadTable);
    } else {
      SearchItem it;
      it.q = a.q + g.q_off * 3;
      it.perm_q = a.perm_q + g.q_off;
      it.rec = crec + c.p_off * kRecLen;
      it.pairs = cpairs + c.tile_off * (kTilePoints / 2) * kPairFloats;
      it.tinfo = ctinfo + c.tile_off * kTinfoFloats;
      it.f = a.f + c.p_off * a.F;
      it.f_out = a.f_out + g.q_off * a.F;
      it.w_out = a.w_out + g.e_off;
      it.dists = a.dists + g.e_off;
      it.idxs = a.idxs + g.e_off;
      it.row0 = g.q_off;
      it.adj_count = nullptr;
      it.qseed = nullptr;
      it.tau0 = nullptr;
      it.cell_start = ccell + c.cell_off;
      it.cbox = cbnd + (int64_t)g.cloud * 8;
      it.cbits = c.bits;
      it.Q = g.Q;
      it.P = c.P;
      it.K = g.K;
      it.ntile = c.ntile;
      it.q0 = (item - g.item_off) * QPC;
      it.q1 = min(it.q0 + QPC, g.Q);
      bool ok;
      if (KMAX > 8 && g.K <= 8)
        ok = search_item<8, WPC, QPW>(a, it, smem, ntp_cap, uses);
      else if (KMAX > 16 && g.K <= 16)
        ok = search_item<(KMAX > 16 ? 16 : KMAX), WPC, QPW>(a, it, smem, ntp_cap, uses);
      else
        ok = search_item<KMAX, WPC, QPW>(a, it, smem, ntp_cap, uses);
      if (!ok) break;
    }
    __syncthreads();  // the next item reuses shared memory (and s_item)
  }
}

// ------------------------------------------------------------------ host

int num_sms(int dev) {
  static int cache[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cache[dev] = v;
  }
  return cache[dev];
}

namespace {

template <int KMAX, int WPC, int QPW>
int launch_search_t(const SearchParams& a, cudaStream_t st) {
  const size_t smem = search_smem_bytes(WPC, QPW) + search_region_c_bytes(a.ntile);
  if (smem > 227 * 1024) return KNNAG_ERR_TOO_LARGE;
  static int attr_set[64] = {0};  // largest size already allowed, per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && attr_set[dev] < (int)smem) {
    if (cudaFuncSetAttribute(search_f32_kernel<KMAX, WPC, QPW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return KNNAG_ERR_CUDA;
    attr_set[dev] = (int)smem;
  }
  constexpr int QPC = WPC * QPW;
  const int nb = (a.Q + QPC - 1) / QPC;
  dim3 grid(nb, a.B);
  const int64_t nbt = (int64_t)nb * a.B;
  bool plan = false;
  if (a.items && nbt <= kPlanMaxBlocks) {
    // the plan pays when the blocks take more than one wave of the search
    static int occ_smem[64], occ_val[64];
    int occ = 0;
    if (dev >= 0 && dev < 64 && occ_smem[dev] == (int)smem) {
      occ = occ_val[dev];
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_f32_kernel<KMAX, WPC, QPW>, 32 * WPC, smem) !=
          cudaSuccess)
        return KNNAG_ERR_CUDA;
      if (dev >= 0 && dev < 64) {
        occ_smem[dev] = (int)smem;
        occ_val[dev] = occ;
      }
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    plan = nbt > (int64_t)occ * sms;
  }
  if (plan) {
    grid = dim3((unsigned)nbt, 1);
    static int items_smem[64];
    if (dev >= 0 && dev < 64 && items_smem[dev] < kPlanMaxBlocks * 4) {
      if (cudaFuncSetAttribute(search_items_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPlanMaxBlocks * 4) != cudaSuccess)
        return KNNAG_ERR_CUDA;
      items_smem[dev] = kPlanMaxBlocks * 4;
    }
  }
  SearchParams ap = a;
  if (!plan) ap.items = nullptr;  // one wave (or too many blocks to plan): the plain grid
  profile_begin(st);  // the plan does the seed work of the search: timed with it
  if (plan) {
    search_plan_kernel<KMAX><<<dim3(nb, a.B), 32 * ((QPC + kPlanQPW - 1) / kPlanQPW), 0, st>>>(ap, QPC, nb);
    search_items_kernel<<<1, kPlanItemsThreads, (size_t)nbt * 4, st>>>(ap, nb, QPC);
    note_launches(2);
  }
  search_f32_kernel<KMAX, WPC, QPW><<<grid, 32 * WPC, smem, st>>>(ap);
  profile_end(st);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template <int KMAX, int WPC, int QPW>
int launch_search_ragged_t(const SearchParams& a, int64_t cap_items, cudaStream_t st) {
  const size_t smem = search_smem_bytes(WPC, QPW) + search_region_c_bytes(a.ntile);
  if (smem > 227 * 1024) return KNNAG_ERR_TOO_LARGE;
  int dev = 0;
  cudaGetDevice(&dev);
  static int attr_set[64] = {0};
  if (dev >= 0 && dev < 64 && attr_set[dev] < (int)smem) {
    if (cudaFuncSetAttribute(search_ragged_kernel<KMAX, WPC, QPW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return KNNAG_ERR_CUDA;
    attr_set[dev] = (int)smem;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search_ragged_kernel<KMAX, WPC, QPW>, 32 * WPC, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int64_t grid = (int64_t)num_sms(dev) * per_sm;
  if (grid > cap_items) grid = cap_items;
  if (grid < 1) grid = 1;
  profile_begin(st);
  search_ragged_kernel<KMAX, WPC, QPW><<<(unsigned)grid, 32 * WPC, smem, st>>>(a);
  profile_end(st);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

// launch-shape code s -> (warps per CTA, queries per warp)
template <int KMAX>
int launch_search_ragged_k(const SearchParams& a, int s, int64_t cap_items, cudaStream_t st) {
  switch (s) {
    case 1: return launch_search_ragged_t<KMAX, 4, 32>(a, cap_items, st);
    case 2: return launch_search_ragged_t<KMAX, 2, 32>(a, cap_items, st);
    case 8: return launch_search_ragged_t<KMAX, 2, 16>(a, cap_items, st);
    case 16: return launch_search_ragged_t<KMAX, 4, 8>(a, cap_items, st);
    case 32: return launch_search_ragged_t<KMAX, 1, 16>(a, cap_items, st);
    case 64: return launch_search_ragged_t<KMAX, 1, 8>(a, cap_items, st);
    default: return launch_search_ragged_t<KMAX, 1, 32>(a, cap_items, st);
  }
}

template <int KMAX>
int launch_search_k(const SearchParams& a, int s, cudaStream_t st) {
  switch (s) {
    case 1: return launch_search_t<KMAX, 4, 32>(a, st);
    case 2: return launch_search_t<KMAX, 2, 32>(a, st);
    case 8: return launch_search_t<KMAX, 2, 16>(a, st);
    case 16: return launch_search_t<KMAX, 4, 8>(a, st);
    case 32: return launch_search_t<KMAX, 1, 16>(a, st);
    case 64: return launch_search_t<KMAX, 1, 8>(a, st);
    default: return launch_search_t<KMAX, 1, 32>(a, st);
  }
}

// Launch shape of the CUDA-core uniform search, by the warps the query set
// gives at 32 queries per warp: many (large query sets) -> 128-query CTAs of
// 4 warps; few -> fewer queries per warp, so that there are more warps to
// hide the latency of each one's dependent work.
int choose_cuda_core_splits(int B, int Q, int dev) {
  const int64_t warps32 = ((int64_t)B * Q + 31) / 32;
  const int64_t sms = num_sms(dev);
  if (warps32 >= 16 * sms) return 1;
  if (warps32 >= 4 * sms) return 8;
  return 16;
}

// The process-wide setting when one is made; else the tensor-core filtered
// search for grids of more than 8 waves of its 128-query CTAs (two per SM),
// where it measured faster (B200, one cloud of 131072 points and 524288
// queries: 2.80 against 2.95 ms), and the CUDA-core search below that (the
// table workload, B = 2, Q = 12288, P = 4096: 0.148 against 0.113 ms).
int choose_splits(int B, int Q, int dev) {
  const int forced = search_splits_setting();
  if (search_setting_ok(forced)) return forced;
  const int64_t ctas = (int64_t)B * ((Q + 127) / 128);
  if (ctas > 16 * (int64_t)num_sms(dev)) return kShapeTensorFilter;
  return choose_cuda_core_splits(B, Q, dev);
}

inline unsigned grid_for(int64_t n, int threads, int dev) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)num_sms(dev) * 32;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

int search_plan_max_blocks() { return kPlanMaxBlocks; }

int launch_search_plan(const SearchParams& a, int qpc, int nb, cudaStream_t st) {
  const int64_t nbt = (int64_t)nb * a.B;
  if (nbt > kPlanMaxBlocks || !a.items || !a.tau0 || !a.plan_est) return KNNAG_ERR_ARG;
  int dev = 0;
  cudaGetDevice(&dev);
  static int items_smem[64];
  if (dev >= 0 && dev < 64 && items_smem[dev] < kPlanMaxBlocks * 4) {
    if (cudaFuncSetAttribute(search_items_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPlanMaxBlocks * 4) !=
        cudaSuccess)
      return KNNAG_ERR_CUDA;
    items_smem[dev] = kPlanMaxBlocks * 4;
  }
  const dim3 grid((unsigned)nb, (unsigned)a.B);
  const unsigned threads = 32 * ((qpc + kPlanQPW - 1) / kPlanQPW);
  if (a.K <= 8)
    search_plan_kernel<8><<<grid, threads, 0, st>>>(a, qpc, nb);
  else if (a.K <= 16)
    search_plan_kernel<16><<<grid, threads, 0, st>>>(a, qpc, nb);
  else
    search_plan_kernel<32><<<grid, threads, 0, st>>>(a, qpc, nb);
  search_items_kernel<<<1, kPlanItemsThreads, (size_t)nbt * 4, st>>>(a, nb, qpc);
  note_launches(2);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template <typename T>
int launch_exact(const ExactParams<T>& a, cudaStream_t st) {
  const size_t smem = (size_t)replay_chunk<T>() * sizeof(T) + (size_t)a.K * (sizeof(T) + sizeof(int));
  if (smem > 200 * 1024) return KNNAG_ERR_TOO_LARGE;
  // A list of flagged queries is short: 512 threads per CTA, fifteen warps
  // computing keys beside the warp that runs MinK.  Every query of a call:
  // 256 threads, more queries per SM at once.
  auto kernel = a.use_list ? mink_replay_kernel<T, 2 * kReplayThreads> : mink_replay_kernel<T, kReplayThreads>;
  const int threads = a.use_list ? 2 * kReplayThreads : kReplayThreads;
  if (smem > 48 * 1024 && cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                              cudaSuccess)
    return KNNAG_ERR_CUDA;
  int dev = 0;
  cudaGetDevice(&dev);
  int64_t blocks;
  if (a.use_list) {
    blocks = (int64_t)num_sms(dev) * 2;  // flagged queries are few; each CTA loops over them
  } else {
    blocks = (int64_t)a.B * a.Q;
    const int64_t cap = (int64_t)num_sms(dev) * 8;
    if (blocks > cap) blocks = cap;
  }
  if (blocks < 1) blocks = 1;
  if (!a.use_list) profile_begin(st);
  kernel<<<(unsigned)blocks, threads, smem, st>>>(a);
  if (!a.use_list) profile_end(st);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template int launch_exact<float>(const ExactParams<float>&, cudaStream_t);
template int launch_exact<double>(const ExactParams<double>&, cudaStream_t);

FwdLayout fwd_layout(int B, int Q, int P, int K, int dtype, bool own_rec) {
  FwdLayout L{};
  const size_t esz = dtype == KNNAG_F64 ? 8 : 4;
  size_t off = 0;
  L.status = off;
  off += 256;
  L.flag_list = off;
  off += align256((size_t)B * Q * 4);
  L.rec = off;
  if (own_rec) off += align256((size_t)B * P * kRecLen * esz);
  L.P_pad = (int)round_up(P, kTilePoints);
  L.pairs = L.bounds = L.cell_count = L.cell_offset = L.perm_p = L.perm_q = L.tinfo = L.qseed = L.tau0 =
      L.plan_est = L.items = L.tcops = L.tcinfo = off;
  L.bits = 0;
  if (dtype == KNNAG_F32 && K <= 32) {
    L.bits = spatial_bits(P);
    const size_t cells = (size_t)1 << (3 * L.bits);
    L.pairs = off;
    off += align256((size_t)B * L.P_pad * kRecLen * 4);
    L.bounds = off;  // per element kBoundParts partial boxes
    off += align256((size_t)B * kBoundParts * 8 * 4);
    // point and query cells of each batch element, sorted together
    L.cell_count = off;
    off += align256(2 * (size_t)B * cells * 4);
    L.cell_offset = off;
    off += align256((2 * (size_t)B * cells + 1) * 4);
    L.perm_p = off;  // perm_q follows perm_p without a gap (one scatter fills both)
    L.perm_q = off + (size_t)B * P * 4;
    off += align256((size_t)B * P * 4 + (size_t)B * Q * 4);
    L.tinfo = off;
    off += align256((size_t)B * (L.P_pad / kTilePoints) * kTinfoBytes);
    L.qseed = off;
    off += align256((size_t)B * Q * 4);
    // search plan: seed thresholds, per-block estimates, CTA items (for the
    // smallest blocks, 8 queries)
    const size_t nb_max = (size_t)B * ((Q + 7) / 8);
    L.tau0 = off;
    off += align256((size_t)B * Q * 4);
    L.plan_est = off;
    off += align256(nb_max * 4);
    L.items = off;
    off += align256(nb_max * 16);
    // tensor-core filter: B operands and bound terms of every tile
    const size_t ntiles = (size_t)B * (L.P_pad / kTilePoints);
    L.tcops = off;
    off += align256(ntiles * kTcOpsBytes);
    L.tcinfo = off;
    off += align256(ntiles * kTcInfoBytes);
  }
  L.total = off;
  return L;
}

int launch_pack_points_bounded(const float* p, const float* sigma, const float* R, int B, int P, float* rec,
                               float* parts, cudaStream_t st, int* zero_words, int n_zero, int* zero_rows,
                               int* zero_cells, int64_t n_cells) {
  pack_points_bounded_kernel<<<dim3(kBoundParts, B), 256, 0, st>>>(p, sigma, R, P, rec, parts, zero_words, n_zero,
                                                                   zero_rows, zero_cells, n_cells);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

int launch_pack_points(const void* p, const void* sigma, const void* R, int B, int P, int dtype, void* rec,
                       cudaStream_t st, int* zero_words, int n_zero, int* zero_rows) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int64_t n = (int64_t)B * P;
  if (dtype == KNNAG_F64)
    pack_points_kernel<double><<<grid_for(n, 256, dev), 256, 0, st>>>(
        (const double*)p, (const double*)sigma, (const double*)R, n, (double*)rec, zero_words, n_zero, zero_rows);
  else
    pack_points_kernel<float><<<grid_for(n, 256, dev), 256, 0, st>>>((const float*)p, (const float*)sigma,
                                                                     (const float*)R, n, (float*)rec, zero_words,
                                                                     n_zero, zero_rows);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template <typename T>
static int forward_exact_all(const T* q, const T* rec, const T* f, int B, int Q, int P, int F, int K, T* f_out,
                             T* w_out, T* dists, int64_t* idxs, int* adj_count, cudaStream_t st) {
  ExactParams<T> e{q, rec, f, nullptr, nullptr, 0, B, Q, P, F, K, 0, nullptr, nullptr, f_out, w_out, dists, idxs};
  e.adj_count = adj_count;
  return launch_exact<T>(e, st);
}

int forward_impl(const void* q, const void* p, const void* f, const void* sigma, const void* R, int B, int Q,
                 int P, int F, int K, int dtype, void* f_out, void* w_out, void* dists, int64_t* idxs,
                 void* points, void* workspace, cudaStream_t st, void* adjacency) {
  NvtxRange range("knnag:forward");
  int* adj_count = adjacency ? reinterpret_cast<int*>(static_cast<char*>(adjacency) + adj_layout(B, Q, P, K).cursor)
                             : nullptr;
  const bool own_rec = points == nullptr;
  const FwdLayout L = fwd_layout(B, Q, P, K, dtype, own_rec);
  char* ws = static_cast<char*>(workspace);
  int* status = reinterpret_cast<int*>(ws + L.status);
  int* flag_count = status + 1;
  int* flag_list = reinterpret_cast<int*>(ws + L.flag_list);
  void* rec = own_rec ? (void*)(ws + L.rec) : points;
  int rc;
  const bool search_path = dtype == KNNAG_F32 && K <= 32;
  {
    NvtxRange r("knnag:pack_points");
    // also zeroes the status words and the adjacency's entry counts; on
    // the search path also the cell counts, and it bounds the points
    if (search_path)
      // cell counts and offsets (the offsets are the scatter's cursors when
      // the scan is folded into it) are zeroed, padding between them included
      rc = launch_pack_points_bounded((const float*)p, (const float*)sigma, (const float*)R, B, P, (float*)rec,
                                      reinterpret_cast<float*>(ws + L.bounds), st, status, 2, adj_count,
                                      reinterpret_cast<int*>(ws + L.cell_count),
                                      (int64_t)(L.cell_offset - L.cell_count) / 4 + (2 * (int64_t)B << (3 * L.bits)) + 1);
    else
      rc = launch_pack_points(p, sigma, R, B, P, dtype, rec, st, status, 2, adj_count);
  }
  if (rc) return rc;
  if (dtype == KNNAG_F64)
    return forward_exact_all<double>((const double*)q, (const double*)rec, (const double*)f, B, Q, P, F, K,
                                     (double*)f_out, (double*)w_out, (double*)dists, idxs, adj_count, st);
  if (K > 32)
    return forward_exact_all<float>((const float*)q, (const float*)rec, (const float*)f, B, Q, P, F, K,
                                    (float*)f_out, (float*)w_out, (float*)dists, idxs, adj_count, st);
  int dev = 0;
  cudaGetDevice(&dev);
  float* pairs = reinterpret_cast<float*>(ws + L.pairs);
  int G = choose_splits(B, Q, dev);
  if (G == kShapeTensorFilter && !search_tc_fits(L.P_pad / kTilePoints)) G = choose_cuda_core_splits(B, Q, dev);
  {
    NvtxRange r("knnag:spatial_index");
    rc = launch_spatial_index((const float*)q, (const float*)rec, B, Q, P, L.P_pad, ws, L, st,
                              G == kShapeTensorFilter);
  }
  if (rc) return rc;
  SearchParams sp{};
  sp.q = (const float*)q;
  sp.perm_q = reinterpret_cast<const int*>(ws + L.perm_q);
  sp.tinfo = reinterpret_cast<const float*>(ws + L.tinfo);
  sp.ntile = L.P_pad / kTilePoints;
  sp.pairs = pairs;
  sp.rec = (const float*)rec;
  sp.f = (const float*)f;
  sp.B = B;
  sp.Q = Q;
  sp.P = P;
  sp.P_pad = L.P_pad;
  sp.F = F;
  sp.K = K;
  sp.vec4 = (F % 4 == 0) && ((uintptr_t)f % 16 == 0) && ((uintptr_t)f_out % 16 == 0);
  sp.f_out = (float*)f_out;
  sp.w_out = (float*)w_out;
  sp.dists = (float*)dists;
  sp.idxs = idxs;
  sp.status = status;
  sp.flag_count = flag_count;
  sp.flag_list = flag_list;
  sp.adj_count = adj_count;
  sp.qseed = reinterpret_cast<const int*>(ws + L.qseed);
  sp.tau0 = reinterpret_cast<float*>(ws + L.tau0);
  sp.plan_est = reinterpret_cast<int*>(ws + L.plan_est);
  sp.items = reinterpret_cast<int4*>(ws + L.items);
  sp.tcops = reinterpret_cast<const float*>(ws + L.tcops);
  sp.tcinfo = reinterpret_cast<const float*>(ws + L.tcinfo);
  apply_search_debug(sp);
  if (G == kShapeTensorFilter) {
    NvtxRange r("knnag:search_tc");
    rc = launch_search_tc(sp, st);
  } else {
    NvtxRange r("knnag:search");
    if (K <= 8)
      rc = launch_search_k<8>(sp, G, st);
    else if (K <= 16)
      rc = launch_search_k<16>(sp, G, st);
    else
      rc = launch_search_k<32>(sp, G, st);
  }
  if (rc) return rc;
  // Exact MinK replay of the flagged queries (count read on the device).
  NvtxRange r("knnag:replay_flagged");
  ExactParams<float> e{(const float*)q, (const float*)rec, (const float*)f, nullptr, nullptr, 0, B, Q, P, F, K, 1,
                       flag_list, flag_count, (float*)f_out, (float*)w_out, (float*)dists, idxs};
  e.adj_count = adj_count;
  return launch_exact<float>(e, st);
}

RaggedLayout ragged_layout(int cap_segs, int64_t cap_q) {
  RaggedLayout L{};
  L.cap_cells = cap_q + 8 * (int64_t)cap_segs;
  size_t off = 0;
  L.status = off;
  off += 256;
  L.flag_list = off;
  off += align256((size_t)cap_q * 4);
  L.perm_q = off;
  off += align256((size_t)cap_q * 4);
  L.cell_count = off;
  off += align256((size_t)L.cap_cells * 4);
  L.cell_offset = off;
  off += align256(((size_t)L.cap_cells + 1) * 4);
  L.total = off;
  return L;
}

// Ragged forward: validate the table, sort every segment's queries, one
// persistent search launch over all segments with K <= 32, exact replay of
// the flagged queries, and the exact kernel for segments with K > 32.
int ragged_forward_impl(const char* cs, const void* segs, const float* q, const float* f, int F, int cap_segs,
                        int64_t cap_q, int64_t cap_e, int max_k, int ntile_cap, int splits, float* f_out, float* w_out,
                        float* dists, int64_t* idxs, void* workspace, cudaStream_t st) {
  NvtxRange range("knnag:ragged_forward");
  const RaggedLayout L = ragged_layout(cap_segs, cap_q);
  char* ws = static_cast<char*>(workspace);
  int* status = reinterpret_cast<int*>(ws + L.status);
  int* flag_count = status + 1;
  int* item_counter = status + 2;
  int* flag_list = reinterpret_cast<int*>(ws + L.flag_list);
  int* perm_q = reinterpret_cast<int*>(ws + L.perm_q);
  const int G = splits;
  const int qpc = search_qpc(G);
  if (cudaMemsetAsync(status, 0, 4 * sizeof(int), st) != cudaSuccess) return KNNAG_ERR_CUDA;
  int rc = launch_validate_segments(cs, segs, cap_segs, cap_q, cap_e, max_k, ntile_cap, qpc, status, st);
  if (rc) return rc;
  rc = launch_query_order(q, cs, segs, cap_segs, cap_q, (int)L.cap_cells, reinterpret_cast<int*>(ws + L.cell_count),
                          reinterpret_cast<int*>(ws + L.cell_offset), perm_q, status, st);
  if (rc) return rc;
  const int ks = max_k < 32 ? max_k : 32;
  SearchParams sp{};
  sp.q = q;
  sp.perm_q = perm_q;
  sp.ntile = ntile_cap;
  sp.f = f;
  sp.B = 1;
  sp.F = F;
  sp.K = ks;
  sp.vec4 = (F % 4 == 0) && ((uintptr_t)f % 16 == 0) && ((uintptr_t)f_out % 16 == 0);
  sp.f_out = f_out;
  sp.w_out = w_out;
  sp.dists = dists;
  sp.idxs = idxs;
  sp.status = status;
  sp.flag_count = flag_count;
  sp.flag_list = flag_list;
  sp.cs = cs;
  sp.segs = segs;
  sp.item_counter = item_counter;
  apply_search_debug(sp);
  const int64_t cap_items = cap_q / qpc + cap_segs;
  if (ks <= 8)
    rc = launch_search_ragged_k<8>(sp, G, cap_items, st);
  else if (ks <= 16)
    rc = launch_search_ragged_k<16>(sp, G, cap_items, st);
  else
    rc = launch_search_ragged_k<32>(sp, G, cap_items, st);
  if (rc) return rc;
  ExactParams<float> e{};
  e.q = q;
  e.f = f;
  e.B = 1;
  e.Q = (int)(cap_q < (1 << 30) ? cap_q : (1 << 30));
  e.F = F;
  e.K = ks;
  e.use_list = 1;
  e.list = flag_list;
  e.list_count = flag_count;
  e.f_out = f_out;
  e.w_out = w_out;
  e.dists = dists;
  e.idxs = idxs;
  e.cs = cs;
  e.segs = segs;
  e.status = status;
  rc = launch_exact<float>(e, st);
  if (rc || max_k <= 32) return rc;
  e.K = max_k;
  e.use_list = 0;
  return launch_exact<float>(e, st);
}

}  // namespace knnag
