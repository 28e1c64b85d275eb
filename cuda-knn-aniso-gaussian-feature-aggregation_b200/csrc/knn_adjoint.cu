// Backward path: the point -> entry adjacency (CSR) and the first- and
// second-order adjoint kernels.
//
// Replaces csrc/backward.cu:5-121 (first order), csrc/backward.cu:124-328
// (second order, Eikonal) and their launchers csrc/backward.cu:331-455.  The
// reference scatters every point-side gradient with float atomicAdd; here
// each gradient is split into a query-side kernel (one query per half-warp,
// sums over its K neighbours) and a point-side kernel (one point per warp,
// sums over the sorted list of entries that selected it), so every sum has a
// fixed order and results are bit-reproducible.
//
// Notation for one entry e = (b, q, k) with point i = idxs[e]:
//   d = q - p_i, u_a = R_a . d, s = sum_a sigma_a u_a^2, w = exp(-s),
//   v = R^T diag(sigma) u  (so dw/dq = -2 w v),  c = gfo[q] . f[i].
// First order (gradient of <gfo, f_out>):
//   dq += -2 c w v,  dp += 2 c w v,  dsigma_a += -c w u_a^2,
//   dR_am += -2 c w sigma_a u_a d_m,  df[i] += w gfo[q].
// Second order (gradient of <g, dq> with g = grad_grad_q[q]):
//   A = g . v, r_a = R_a . g, Mg = sum_a sigma_a r_a R_a,
//   T = 2 c w (2 A v - Mg): dq += T, dp -= T,
//   dsigma_a += 2 c w u_a (u_a A - r_a),
//   dR_am += -2 c w sigma_a (-2 u_a d_m A + d_m r_a + u_a g_m),
//   df[i] += -2 w A gfo[q],  dgfo[q] += -2 w A f[i].
#include <math.h>

#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {

AdjLayout adj_layout(int B, int Q, int P, int K) {
  AdjLayout L{};
  const size_t n_rows = (size_t)B * P;
  const size_t n = (size_t)B * Q * K;
  size_t off = 0;
  L.rowptr = off;
  off += align256((n_rows + 1) * 4);
  L.cursor = off;
  off += align256(n_rows * 4);
  L.unsorted = off;
  off += align256(n * 4);
  L.entries = off;
  off += align256(n * 4);
  L.total = off;
  return L;
}

// ----------------------------------------------------------------- CSR

__global__ void adj_count_kernel(const int64_t* __restrict__ idxs, int n, int qk, int P, int* __restrict__ count) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int64_t idx = idxs[e];
    if (idx < 0 || idx >= P) continue;  // not a point index: no row holds it
    atomicAdd(&count[(e / qk) * P + (int)idx], 1);
  }
}

// Exclusive scan of count[0..n) into rowptr[0..n] by one CTA of 1024
// threads (4 items per thread per pass); count is zeroed on the way so it
// can serve as the fill cursor.
__global__ void __launch_bounds__(1024) adj_scan_kernel(int* __restrict__ count, int64_t n, int* __restrict__ rowptr) {
  __shared__ int warp_sums[32];
  __shared__ int carry_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry_s = 0;
  __syncthreads();
  for (int64_t base = 0; base < n; base += 4096) {
    int v[4];
    int local = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t i = base + (int64_t)tid * 4 + u;
      v[u] = (i < n) ? count[i] : 0;
      if (i < n) count[i] = 0;
      local += v[u];
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int ws = warp_sums[lane];
      int wi = ws;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      warp_sums[lane] = wi - ws;  // exclusive prefix of warp totals
    }
    __syncthreads();
    int run = carry_s + warp_sums[warp] + incl - local;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t i = base + (int64_t)tid * 4 + u;
      if (i < n) rowptr[i] = run;
      run += v[u];
    }
    __syncthreads();
    if (tid == 1023) carry_s = run;
    __syncthreads();
  }
  if (tid == 0) rowptr[n] = carry_s;
}

// Multi-CTA exclusive scan for long arrays, in three passes over chunks of
// kScanChunk elements (1024 threads x 8): (1) each CTA writes its chunk's
// sum to out[chunk start]; (2) one CTA replaces those sums by their
// exclusive prefix and writes the total to out[n]; (3) each CTA scans its
// chunk from that prefix into out and zeroes count.  The chunk sums live in
// out itself, so no scratch is needed.
constexpr int kScanChunk = 8192;

__device__ __forceinline__ int block_exclusive_scan_1024(int local, int* warp_sums, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int ws = warp_sums[lane];
    int wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_sums[lane] = wi - ws;
    if (lane == 31) warp_sums[32] = wi;
  }
  __syncthreads();
  total = warp_sums[32];
  return warp_sums[warp] + incl - local;
}

__global__ void __launch_bounds__(1024) scan_chunk_sums_kernel(const int* __restrict__ count, int64_t n,
                                                               int* __restrict__ out) {
  __shared__ int warp_sums[33];
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * 8;
  int local = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u)
    if (base + u < n) local += count[base + u];
  int total;
  block_exclusive_scan_1024(local, warp_sums, total);
  if (threadIdx.x == 0) out[(int64_t)blockIdx.x * kScanChunk] = total;
}

__global__ void __launch_bounds__(1024) scan_chunk_prefix_kernel(int* __restrict__ out, int64_t n, int chunks) {
  __shared__ int warp_sums[33];
  __shared__ int carry_s;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int c0 = 0; c0 < chunks; c0 += 1024) {
    const int c = c0 + threadIdx.x;
    const int v = c < chunks ? out[(int64_t)c * kScanChunk] : 0;
    int total;
    const int ex = block_exclusive_scan_1024(v, warp_sums, total);
    if (c < chunks) out[(int64_t)c * kScanChunk] = carry_s + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry_s += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry_s;
}

__global__ void __launch_bounds__(1024) scan_chunk_apply_kernel(int* __restrict__ count, int64_t n,
                                                                int* __restrict__ out) {
  __shared__ int warp_sums[33];
  __shared__ int prefix_s;
  const int64_t chunk0 = (int64_t)blockIdx.x * kScanChunk;
  if (threadIdx.x == 0) prefix_s = out[chunk0];
  const int64_t base = chunk0 + (int64_t)threadIdx.x * 8;
  int v[8];
  int local = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    v[u] = base + u < n ? count[base + u] : 0;
    local += v[u];
  }
  int total;
  int run = block_exclusive_scan_1024(local, warp_sums, total) + prefix_s;  // barriers order the prefix read
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    if (base + u < n) {
      out[base + u] = run;
      count[base + u] = 0;
    }
    run += v[u];
  }
}

__global__ void adj_fill_kernel(const int64_t* __restrict__ idxs, int n, int qk, int P, const int* __restrict__ rowptr,
                                int* __restrict__ cursor, int* __restrict__ unsorted) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int64_t idx = idxs[e];
    if (idx < 0 || idx >= P) continue;
    const int row = (e / qk) * P + (int)idx;
    unsorted[rowptr[row] + atomicAdd(&cursor[row], 1)] = e;
  }
}

// Bitonic sort, ascending, of the 32*V ints of a warp: element lane + 32*h
// sits in x[h].  Stages with a partner distance below 32 exchange through
// shuffles, the others inside the lane.
template <int V>
__device__ __forceinline__ void warp_bitonic_sort(int (&x)[V], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * V; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int h = 0; h < V; ++h) {
          const int hp = h ^ (j >> 5);
          if (hp > h) {
            const bool up = ((32 * h) & k) == 0;  // lane < 32 <= j < k
            const int lo = min(x[h], x[hp]), hi = max(x[h], x[hp]);
            x[h] = up ? lo : hi;
            x[hp] = up ? hi : lo;
          }
        }
      } else {
#pragma unroll
        for (int h = 0; h < V; ++h) {
          const int e = lane + 32 * h;
          const int o = __shfl_xor_sync(0xffffffffu, x[h], j);
          const bool up = (e & k) == 0, lower = (e & j) == 0;
          x[h] = (lower == up) ? min(x[h], o) : max(x[h], o);
        }
      }
    }
  }
}

template <int V>
__device__ __forceinline__ void sort_row_regs(const int* src, int n, int* dst, int lane) {
  int x[V];
#pragma unroll
  for (int h = 0; h < V; ++h) x[h] = lane + 32 * h < n ? src[lane + 32 * h] : 0x7fffffff;
  warp_bitonic_sort<V>(x, lane);
#pragma unroll
  for (int h = 0; h < V; ++h)
    if (lane + 32 * h < n) dst[lane + 32 * h] = x[h];
}

constexpr int kAdjSortWarps = 8;      // warps per CTA of adj_sort_kernel
constexpr int kAdjSmemSort = 1024;    // longest row sorted in shared memory

// Sort every row by entry id, one warp per row (ids in a row are distinct:
// a query selects a point at most once).  Rows of up to 256 entries are
// bitonic-sorted in registers, rows of up to 1024 in the warp's shared
// memory; longer rows place each id at the number of smaller ids in the row.
__global__ void __launch_bounds__(kAdjSortWarps * 32) adj_sort_kernel(const int* __restrict__ rowptr,
                                                                     const int* __restrict__ unsorted, int n_rows,
                                                                     int* __restrict__ entries) {
  __shared__ int sbuf[kAdjSortWarps][kAdjSmemSort];
  const int lane = threadIdx.x & 31;
  int* sb = sbuf[threadIdx.x >> 5];
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int r = gw; r < n_rows; r += nw) {
    const int start = rowptr[r];
    const int n = rowptr[r + 1] - start;
    const int* src = unsorted + start;
    int* dst = entries + start;
    if (n <= 32) {
      sort_row_regs<1>(src, n, dst, lane);
    } else if (n <= 64) {
      sort_row_regs<2>(src, n, dst, lane);
    } else if (n <= 128) {
      sort_row_regs<4>(src, n, dst, lane);
    } else if (n <= 256) {
      sort_row_regs<8>(src, n, dst, lane);
    } else if (n <= kAdjSmemSort) {
      int n2 = 512;
      while (n2 < n) n2 <<= 1;
      for (int i = lane; i < n2; i += 32) sb[i] = i < n ? src[i] : 0x7fffffff;
      __syncwarp();
      for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = lane; i < n2; i += 32) {
            const int ixj = i ^ j;
            if (ixj > i) {
              const int a = sb[i], b = sb[ixj];
              if ((a > b) == ((i & k) == 0)) {
                sb[i] = b;
                sb[ixj] = a;
              }
            }
          }
          __syncwarp();
        }
      }
      for (int i = lane; i < n; i += 32) dst[i] = sb[i];
      __syncwarp();
    } else {
      for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const int v = (i < n) ? src[i] : 0;
        int rank = 0;
        for (int jb = 0; jb < n; jb += 32) {
          const int uj = (jb + lane < n) ? src[jb + lane] : 0x7fffffff;
          const int lim = min(32, n - jb);
          for (int jj = 0; jj < lim; ++jj) {
            const int u = __shfl_sync(0xffffffffu, uj, jj);
            rank += (u < v || (u == v && jb + jj < i)) ? 1 : 0;  // stable even if ids repeat
          }
        }
        if (i < n) dst[rank] = v;
      }
    }
  }
}

namespace {
int sm_count() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
  return v;
}
inline unsigned blocks_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 32;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}
}  // namespace

// Exclusive scan of count[0..n) into out[0..n] (out[n] = total); count is
// zeroed so it can serve as a fill cursor.  One CTA for short arrays, the
// three-pass multi-CTA scan for long ones.
int launch_exclusive_scan(int* count, int n, int* out, cudaStream_t st) {
  if (n <= 4 * kScanChunk) {
    adj_scan_kernel<<<1, 1024, 0, st>>>(count, n, out);
    note_launches(1);
  } else {
    const int chunks = (int)(((int64_t)n + kScanChunk - 1) / kScanChunk);
    scan_chunk_sums_kernel<<<chunks, 1024, 0, st>>>(count, n, out);
    scan_chunk_prefix_kernel<<<1, 1024, 0, st>>>(out, n, chunks);
    scan_chunk_apply_kernel<<<chunks, 1024, 0, st>>>(count, n, out);
    note_launches(3);
  }
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

int launch_build_adjacency(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, cudaStream_t st,
                           bool counted) {
  NvtxRange range("knnag:adjacency");
  const AdjLayout L = adj_layout(B, Q, P, K);
  char* base = static_cast<char*>(adjacency);
  int* rowptr = reinterpret_cast<int*>(base + L.rowptr);
  int* cursor = reinterpret_cast<int*>(base + L.cursor);
  int* unsorted = reinterpret_cast<int*>(base + L.unsorted);
  int* entries = reinterpret_cast<int*>(base + L.entries);
  const int n = B * Q * K, rows = B * P, qk = Q * K;  // sizes checked < 2^31 by the caller
  if (!counted) {  // else the forward counted the entries per row already
    if (cudaMemsetAsync(cursor, 0, (size_t)rows * 4, st) != cudaSuccess) return KNNAG_ERR_CUDA;
    adj_count_kernel<<<blocks_for(n, 256), 256, 0, st>>>(idxs, n, qk, P, cursor);
    note_launches(1);
  }
  const int rc = launch_exclusive_scan(cursor, rows, rowptr, st);
  if (rc) return rc;
  adj_fill_kernel<<<blocks_for(n, 256), 256, 0, st>>>(idxs, n, qk, P, rowptr, cursor, unsorted);
  const int sort_threads = kAdjSortWarps * 32;
  adj_sort_kernel<<<blocks_for((int64_t)rows * 32, sort_threads), sort_threads, 0, st>>>(rowptr, unsorted, rows,
                                                                                       entries);
  note_launches(2);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

// ------------------------------------------------------------ geometry

template <typename T>
struct Geo {
  T d[3], u[3], s, w;
};

// Offset, rotated offset, key and weight of query (qx,qy,qz) against a
// point record, with the forward's exact arithmetic (so w equals w_out).
template <typename T>
__device__ __forceinline__ void geometry(T qx, T qy, T qz, const T* rec, Geo<T>& g) {
  g.d[0] = add_rn(qx, rec[kNPX]);
  g.d[1] = add_rn(qy, rec[kNPY]);
  g.d[2] = add_rn(qz, rec[kNPZ]);
  const T* r = rec + kR00;
#pragma unroll
  for (int a = 0; a < 3; ++a) g.u[a] = row_dot(r[3 * a + 0], r[3 * a + 1], r[3 * a + 2], g.d[0], g.d[1], g.d[2]);
  g.s = quad_form(g.u[0], g.u[1], g.u[2], rec[kS0], rec[kS1], rec[kS2]);
  g.w = weight_of(g.s);
}

template <typename T>
struct QueryParams {
  const T* gfo;
  const T* ggq;
  const T* q;
  const T* rec;
  const T* f;
  const T* w_in;     // optional saved weights
  const int64_t* idxs;
  const T* coef_in;  // optional c = gfo . f (second order)
  int B, Q, P, F, K;
  T* dq;             // optional
  T* coef_out;       // optional (first order)
  T* dgfo;           // optional (second order)
  // ragged first order (FP32): sizes and offsets from the segment table,
  // records from the cloud set; gfo may be null (all ones).  Nothing is done
  // when *status is nonzero (a table that failed validation).
  const char* cs;
  const void* segs;
  const int* status;
  // broadcast grad_f_out: gfo points to one value s, and c = s * frowsum[i]
  // (frowsum = per-point sum over the columns of f)
  const T* frowsum;
};

template <typename T>
struct PointParams {
  const T* gfo;
  const T* ggq;
  const T* q;
  const T* rec;
  const T* w_in;
  const T* coef;
  const int* rowptr;
  const int* entries;
  int B, Q, P, F, K;
  int needs;
  T* dp;
  T* df;
  T* dsigma;
  T* dR;
  bool gfo_scalar;  // gfo points to one value broadcast over [B,Q,F]
};

// v = R^T diag(sigma) u
template <typename T>
__device__ __forceinline__ void rot_back(const T* r, const T* sg, const T* u, T* v) {
#pragma unroll
  for (int m = 0; m < 3; ++m) v[m] = sg[0] * u[0] * r[m] + sg[1] * u[1] * r[3 + m] + sg[2] * u[2] * r[6 + m];
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Per-point sum over the columns of f (one warp per row, fixed reduction
// order): with a broadcast grad_f_out s, c = gfo[q] . f[i] = s * rowsum[i].
// knnag_feature_row_sums exposes the same kernel, so row sums a caller
// keeps for resident features match the ones a backward call computes.
template <typename T>
__global__ void __launch_bounds__(256) row_sum_kernel(const T* __restrict__ f, int64_t rows, int F,
                                                      T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t r = gw; r < rows; r += nw) {
    T acc = T(0);
    for (int c = lane; c < F; c += 32) acc += f[r * F + c];
    acc = warp_sum(acc);
    if (lane == 0) out[r] = acc;
  }
}

// First-order query side with a broadcast grad_f_out s: c_k = s *
// rowsum(f)[idx_k] needs no F-wide dot product, so each lane takes one
// neighbour, and a warp serves two queries when K <= 16 (uniform calls).
template <typename T>
__device__ __forceinline__ void query_order1_scalar(const QueryParams<T>& a, const SegHeader* sh, int64_t BQ) {
  const int lane = threadIdx.x & 31;
  const int lpq = (!sh && a.K <= 16) ? 16 : 32;  // lanes per query
  const int qpw = 32 / lpq, sub = lane / lpq, kl = lane % lpq;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  const T sg0 = a.gfo ? a.gfo[0] : T(1);  // ragged calls: no grad_f_out means all ones
  for (int64_t base = gw * qpw; base < BQ; base += nw * qpw) {
    const int64_t bq = base + sub;
    T acc[3] = {T(0), T(0), T(0)};
    if (bq < BQ) {
      int K, P;
      int64_t e0, pbase;
      const T* recb;
      if (sh) {
        const SegDesc* sd = seg_descs(a.segs);
        const SegDesc g = sd[seg_of_row(sd, sh->nseg, bq)];
        const CloudDesc c = cloud_descs(a.cs)[g.cloud];
        K = g.K;
        P = c.P;
        e0 = g.e_off + (bq - g.q_off) * K;
        pbase = c.p_off;
        recb = reinterpret_cast<const T*>(a.cs + reinterpret_cast<const CloudSetHeader*>(a.cs)->rec_off) +
               c.p_off * kRecLen;
      } else {
        const int64_t b = bq / a.Q;
        K = a.K;
        P = a.P;
        e0 = bq * K;
        pbase = b * a.P;
        recb = a.rec + b * a.P * kRecLen;
      }
      const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];
      for (int k = kl; k < K; k += lpq) {
        const int64_t e = e0 + k;
        const int64_t idx = a.idxs[e];
        T c = T(0);
        if (idx >= 0 && idx < P) {
          c = sg0 * a.frowsum[pbase + idx];
          T rr[kRecLen];
          load_rec(recb + idx * kRecLen, rr);
          const T* rec = rr;
          Geo<T> geo;
          geometry(qx, qy, qz, rec, geo);
          const T w = a.w_in ? a.w_in[e] : geo.w;
          const T sg[3] = {rec[kS0], rec[kS1], rec[kS2]};
          T v[3];
          rot_back(rec + kR00, sg, geo.u, v);
          const T t = T(-2) * c * w;
#pragma unroll
          for (int mm = 0; mm < 3; ++mm) acc[mm] += t * v[mm];
        }
        if (a.coef_out) a.coef_out[e] = c;
      }
    }
#pragma unroll
    for (int mm = 0; mm < 3; ++mm)
      for (int o = lpq >> 1; o >= 1; o >>= 1) acc[mm] += __shfl_xor_sync(0xffffffffu, acc[mm], o);
    if (bq < BQ && kl == 0 && a.dq) {
      a.dq[bq * 3 + 0] = acc[0];
      a.dq[bq * 3 + 1] = acc[1];
      a.dq[bq * 3 + 2] = acc[2];
    }
  }
}

// First-order query side: one warp per query.  For each group of 8
// neighbours the lanes sweep the feature columns (coalesced rows of f, all
// 8 rows in flight), then a reduce-scatter leaves c_k = gfo[q] . f[idx_k] of
// neighbour k0 + (lane >> 2) in lanes 4m..4m+3; the first lane of each quad
// does that neighbour's geometry.  dq = sum_k -2 c_k w_k v_k.
template <typename T>
__global__ void __launch_bounds__(256, 3) query_order1_kernel(QueryParams<T> a) {
  constexpr int NG = 8;
  const int lane = threadIdx.x & 31;
  const int F = a.F;
  const SegHeader* sh = static_cast<const SegHeader*>(a.segs);
  if (sh && *a.status) return;
  const int64_t BQ = sh ? sh->grad_rows : (int64_t)a.B * a.Q;
  if (a.frowsum) {
    query_order1_scalar(a, sh, BQ);
    return;
  }
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (gridDim.x * (int64_t)blockDim.x) >> 5;
  for (int64_t bq = gw; bq < BQ; bq += nw) {
    // the query's cloud: records, features, sizes and first entry
    int K, P;
    int64_t e0;
    const T* recb;
    const T* fb;
    if (sh) {
      const SegDesc* sd = seg_descs(a.segs);
      const SegDesc g = sd[seg_of_row(sd, sh->nseg, bq)];
      const CloudDesc c = cloud_descs(a.cs)[g.cloud];
      K = g.K;
      P = c.P;
      e0 = g.e_off + (bq - g.q_off) * K;
      recb = reinterpret_cast<const T*>(a.cs + reinterpret_cast<const CloudSetHeader*>(a.cs)->rec_off) +
             c.p_off * kRecLen;
      fb = a.f + c.p_off * F;
    } else {
      const int64_t b = bq / a.Q;
      K = a.K;
      P = a.P;
      e0 = bq * K;
      recb = a.rec + b * a.P * kRecLen;
      fb = a.f + b * a.P * F;
    }
    const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];
    const T* grow = a.gfo ? a.gfo + bq * F : nullptr;
    T acc[3] = {T(0), T(0), T(0)};
    for (int k0 = 0; k0 < K; k0 += NG) {
      const int nk = min(NG, K - k0);
      int ik[NG];  // neighbour point index within the batch, -1 if none
#pragma unroll
      for (int kk = 0; kk < NG; ++kk) {
        const int64_t idx = kk < nk ? a.idxs[e0 + k0 + kk] : -1;
        ik[kk] = (idx >= 0 && idx < P) ? (int)idx : -1;
      }
      T part[NG];
#pragma unroll
      for (int kk = 0; kk < NG; ++kk) part[kk] = T(0);
      for (int c = lane; c < F; c += 32) {
        const T g = grow ? grow[c] : T(1);
#pragma unroll
        for (int kk = 0; kk < NG; ++kk)
          if (ik[kk] >= 0) part[kk] = fma_rn(g, fb[(int64_t)ik[kk] * F + c], part[kk]);
      }
      // reduce-scatter: 8 values over 32 lanes -> lane holds value (lane >> 2) & 7
#pragma unroll
      for (int h = NG / 2, m = 16; h >= 1; h >>= 1, m >>= 1) {
        const bool upper = (lane & m) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
          const T send = upper ? part[i] : part[i + h];
          const T keep = upper ? part[i + h] : part[i];
          part[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
      }
      T c_own = part[0] + __shfl_xor_sync(0xffffffffu, part[0], 2);
      c_own += __shfl_xor_sync(0xffffffffu, c_own, 1);
      const int m_own = lane >> 2;
      const int64_t e = e0 + k0 + m_own;
      if ((lane & 3) == 0 && m_own < nk) {
        if (a.coef_out) a.coef_out[e] = c_own;
        const int64_t idx = a.idxs[e];
        if (idx >= 0 && idx < P) {
          T rr[kRecLen];
          load_rec(recb + idx * kRecLen, rr);
          const T* rec = rr;
          Geo<T> geo;
          geometry(qx, qy, qz, rec, geo);
          const T w = a.w_in ? a.w_in[e] : geo.w;
          const T sg[3] = {rec[kS0], rec[kS1], rec[kS2]};
          T v[3];
          rot_back(rec + kR00, sg, geo.u, v);
          const T t = T(-2) * c_own * w;
#pragma unroll
          for (int mm = 0; mm < 3; ++mm) acc[mm] += t * v[mm];
        }
      }
    }
#pragma unroll
    for (int mm = 0; mm < 3; ++mm) acc[mm] = warp_sum(acc[mm]);
    if (lane == 0 && a.dq) {
      a.dq[bq * 3 + 0] = acc[0];
      a.dq[bq * 3 + 1] = acc[1];
      a.dq[bq * 3 + 2] = acc[2];
    }
  }
}

// Second-order query side: one warp per query, lane = neighbour.  With
// g = grad_grad_q[q], A = g . v, r_a = R_a . g, Mg = sum_a sigma_a r_a R_a:
// dq += 2 c w (2 A v - Mg); optionally dgfo[q] = sum_k (-2 w_k A_k) f[idx_k]
// accumulated in k order, lanes spanning columns, 8 rows in flight.
// Second order without dgfo and with K <= 16 (the Eikonal step): half a
// warp per query, one neighbour per lane, so a warp serves two queries.
template <typename T>
__device__ __forceinline__ void query_order2_half(const QueryParams<T>& a, int64_t blk, int64_t nblk) {
  const int lane = threadIdx.x & 31;
  const int sub = lane >> 4, k = lane & 15;
  const int64_t BQ = (int64_t)a.B * a.Q;
  const int K = a.K, P = a.P;
  const int64_t gw = (blk * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (nblk * (int64_t)blockDim.x) >> 5;
  for (int64_t base = gw * 2; base < BQ; base += nw * 2) {
    const int64_t bq = base + sub;
    T acc[3] = {T(0), T(0), T(0)};
    if (bq < BQ && k < K && a.coef_in) {
      const int64_t b = bq / a.Q;
      const int64_t e = bq * K + k;
      const int64_t idx = a.idxs[e];
      if (idx >= 0 && idx < P) {
        const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];
        const T g[3] = {a.ggq[bq * 3 + 0], a.ggq[bq * 3 + 1], a.ggq[bq * 3 + 2]};
        T rr[kRecLen];
        load_rec(a.rec + (b * P + idx) * kRecLen, rr);
        const T* rec = rr;
        Geo<T> geo;
        geometry(qx, qy, qz, rec, geo);
        const T w = a.w_in ? a.w_in[e] : geo.w;
        const T* r = rec + kR00;
        const T sg[3] = {rec[kS0], rec[kS1], rec[kS2]};
        T v[3];
        rot_back(r, sg, geo.u, v);
        const T A = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
        T rg[3];
#pragma unroll
        for (int s2 = 0; s2 < 3; ++s2) rg[s2] = r[3 * s2] * g[0] + r[3 * s2 + 1] * g[1] + r[3 * s2 + 2] * g[2];
        const T cw2 = T(2) * a.coef_in[e] * w;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const T mg = sg[0] * rg[0] * r[m] + sg[1] * rg[1] * r[3 + m] + sg[2] * rg[2] * r[6 + m];
          acc[m] += cw2 * (T(2) * A * v[m] - mg);
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int o = 8; o >= 1; o >>= 1) acc[m] += __shfl_xor_sync(0xffffffffu, acc[m], o);
    if (bq < BQ && k == 0 && a.dq) {
      a.dq[bq * 3 + 0] = acc[0];
      a.dq[bq * 3 + 1] = acc[1];
      a.dq[bq * 3 + 2] = acc[2];
    }
  }
}

template <typename T>
__device__ __forceinline__ void query_order2_body(const QueryParams<T>& a, int blk, int nblk) {
  if (!a.dgfo && a.K <= 16) {
    query_order2_half(a, blk, nblk);
    return;
  }
  const int lane = threadIdx.x & 31;
  const int BQ = a.B * a.Q, K = a.K, F = a.F, P = a.P;
  const int gw = (blk * blockDim.x + threadIdx.x) >> 5;
  const int nw = (nblk * blockDim.x) >> 5;
  for (int bq = gw; bq < BQ; bq += nw) {
    const int b = bq / a.Q;
    const T qx = a.q[(int64_t)bq * 3 + 0], qy = a.q[(int64_t)bq * 3 + 1], qz = a.q[(int64_t)bq * 3 + 2];
    const T g[3] = {a.ggq[(int64_t)bq * 3 + 0], a.ggq[(int64_t)bq * 3 + 1], a.ggq[(int64_t)bq * 3 + 2]};
    const T* fb = a.f + (int64_t)b * P * F;
    T acc[3] = {T(0), T(0), T(0)};
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      const int64_t e = (int64_t)bq * K + k;
      T a_own = T(0);
      int64_t row = -1;
      if (k < K) {
        const int64_t idx = a.idxs[e];
        if (idx >= 0 && idx < P) {
          row = idx * F;
          T rr[kRecLen];
          load_rec(a.rec + ((int64_t)b * P + idx) * kRecLen, rr);
          const T* rec = rr;
          Geo<T> geo;
          geometry(qx, qy, qz, rec, geo);
          const T w = a.w_in ? a.w_in[e] : geo.w;
          const T* r = rec + kR00;
          const T sg[3] = {rec[kS0], rec[kS1], rec[kS2]};
          T v[3];
          rot_back(r, sg, geo.u, v);
          const T A = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
          a_own = T(-2) * w * A;
          if (a.coef_in) {
            T rg[3];
#pragma unroll
            for (int s2 = 0; s2 < 3; ++s2) rg[s2] = r[3 * s2] * g[0] + r[3 * s2 + 1] * g[1] + r[3 * s2 + 2] * g[2];
            const T cw2 = T(2) * a.coef_in[e] * w;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              const T mg = sg[0] * rg[0] * r[m] + sg[1] * rg[1] * r[3 + m] + sg[2] * rg[2] * r[6 + m];
              acc[m] += cw2 * (T(2) * A * v[m] - mg);
            }
          }
        }
      }
      if (a.dgfo) {
        const int nk = min(32, K - k0);
        T* drow = a.dgfo + (int64_t)bq * F;
        for (int cb = 0; cb < F; cb += 32) {  // warp-uniform: the shuffles below need every lane
          const int c = cb + lane;
          const bool col = c < F;
          T s = (k0 == 0 || !col) ? T(0) : drow[c];
          for (int j0 = 0; j0 < nk; j0 += 8) {
            T val[8], ak[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const int src = min(j0 + jj, 31);
              const int64_t rj = __shfl_sync(0xffffffffu, row, src);
              ak[jj] = __shfl_sync(0xffffffffu, a_own, src);
              val[jj] = (col && j0 + jj < nk && rj >= 0) ? fb[rj + c] : T(0);
            }
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
              if (j0 + jj < nk) s = fma_rn(ak[jj], val[jj], s);
          }
          if (col) drow[c] = s;
        }
      }
    }
    if (a.dq) {
#pragma unroll
      for (int m = 0; m < 3; ++m) acc[m] = warp_sum(acc[m]);
      if (lane == 0) {
        a.dq[(int64_t)bq * 3 + 0] = acc[0];
        a.dq[(int64_t)bq * 3 + 1] = acc[1];
        a.dq[(int64_t)bq * 3 + 2] = acc[2];
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) query_order2_kernel(QueryParams<T> a) {
  query_order2_body(a, blockIdx.x, gridDim.x);
}

// One warp per point row.  Lane j takes entry j of each 32-entry chunk of
// the row for the per-entry geometry (15 point-side scalars, reduced over
// the warp at the end); for df the warp then walks the chunk four entries at
// a time with lanes spanning feature columns (NCOL per lane, coalesced gfo
// rows, four rows in flight).  The entry order of a row is fixed (sorted),
// so every sum has a fixed order.
template <typename T, int ORDER, int NCOL>
__device__ __forceinline__ void point_side_body(const PointParams<T>& a, int blk, int nblk) {
  const int lane = threadIdx.x & 31;
  const int gw = (blk * blockDim.x + threadIdx.x) >> 5;
  const int nw = (nblk * blockDim.x) >> 5;
  const int rows = a.B * a.P;
  const int F = a.F, K = a.K;
  const int n_entries = a.B * a.Q * K;
  const bool want_geo = (a.needs & (KNNAG_NEED_DP | KNNAG_NEED_DSIGMA | KNNAG_NEED_DR)) != 0;
  const bool want_df = (a.needs & KNNAG_NEED_DF) != 0;
  for (int row = gw; row < rows; row += nw) {
    const T* rec = a.rec + (int64_t)row * kRecLen;
    T pr[kRecLen];
#pragma unroll
    for (int m = 0; m < kRecLen; ++m) pr[m] = rec[m];
    const T* r = pr + kR00;
    const T sg[3] = {pr[kS0], pr[kS1], pr[kS2]};
    const int start = a.rowptr[row], end = a.rowptr[row + 1];
    T gp[3] = {T(0), T(0), T(0)}, gs[3] = {T(0), T(0), T(0)}, gR[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) gR[m] = T(0);
    // broadcast grad_f_out s: df[i][c] = s * sum_e wgt_e for every column
    // (one pass, no gathers of grad_f_out rows); wsum is this lane's share
    T wsum = T(0);
    for (int c0 = 0; c0 == 0 || (want_df && !a.gfo_scalar && c0 < F); c0 += 32 * NCOL) {
      T acc[NCOL];
#pragma unroll
      for (int u = 0; u < NCOL; ++u) acc[u] = T(0);
      for (int base = start; base < end; base += 32) {
        const int j = base + lane;
        int e = (j < end) ? a.entries[j] : -1;
        const bool valid = e >= 0 && e < n_entries;
        if (!valid) e = 0;
        const int bq = e / K;
        T wgt = T(0);
        if (valid) {
          const T qx = a.q[(int64_t)bq * 3 + 0], qy = a.q[(int64_t)bq * 3 + 1], qz = a.q[(int64_t)bq * 3 + 2];
          Geo<T> geo;
          geometry(qx, qy, qz, pr, geo);
          const T w = a.w_in ? a.w_in[e] : geo.w;
          T v[3];
          rot_back(r, sg, geo.u, v);
          const T c = (want_geo && c0 == 0) ? a.coef[e] : T(0);
          if (ORDER == 1) {
            wgt = w;
            if (want_geo && c0 == 0) {
              const T cw = c * w;
#pragma unroll
              for (int m = 0; m < 3; ++m) gp[m] += T(2) * cw * v[m];
#pragma unroll
              for (int s2 = 0; s2 < 3; ++s2) {
                gs[s2] -= cw * geo.u[s2] * geo.u[s2];
                const T t = T(-2) * cw * sg[s2] * geo.u[s2];
#pragma unroll
                for (int m = 0; m < 3; ++m) gR[3 * s2 + m] += t * geo.d[m];
              }
            }
          } else {
            const T g[3] = {a.ggq[(int64_t)bq * 3 + 0], a.ggq[(int64_t)bq * 3 + 1], a.ggq[(int64_t)bq * 3 + 2]};
            const T A = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
            wgt = T(-2) * w * A;
            if (want_geo && c0 == 0) {
              T rg[3];
#pragma unroll
              for (int s2 = 0; s2 < 3; ++s2) rg[s2] = r[3 * s2] * g[0] + r[3 * s2 + 1] * g[1] + r[3 * s2 + 2] * g[2];
              const T cw = c * w;
#pragma unroll
              for (int m = 0; m < 3; ++m) {
                const T mg = sg[0] * rg[0] * r[m] + sg[1] * rg[1] * r[3 + m] + sg[2] * rg[2] * r[6 + m];
                gp[m] -= T(2) * cw * (T(2) * A * v[m] - mg);
              }
#pragma unroll
              for (int s2 = 0; s2 < 3; ++s2) {
                gs[s2] += T(2) * cw * geo.u[s2] * (geo.u[s2] * A - rg[s2]);
                const T t = T(-2) * cw * sg[s2];
#pragma unroll
                for (int m = 0; m < 3; ++m)
                  gR[3 * s2 + m] += t * (T(-2) * geo.u[s2] * geo.d[m] * A + geo.d[m] * rg[s2] + geo.u[s2] * g[m]);
              }
            }
          }
        }
        if (want_df && a.gfo_scalar) {
          wsum += wgt;  // 0 for lanes without an entry
        } else if (want_df) {
          const int nvalid = min(32, end - base);
          for (int j0 = 0; j0 < nvalid; j0 += 4) {
            T val[4][NCOL], wj[4];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
              const int src = min(j0 + jj, 31);
              const int bqj = __shfl_sync(0xffffffffu, bq, src);
              wj[jj] = (j0 + jj < nvalid) ? __shfl_sync(0xffffffffu, wgt, src) : T(0);
              const T* grow = a.gfo + (int64_t)bqj * F;
#pragma unroll
              for (int u = 0; u < NCOL; ++u) {
                const int cc = c0 + lane + 32 * u;
                val[jj][u] = (cc < F) ? grow[cc] : T(0);
              }
            }
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
#pragma unroll
              for (int u = 0; u < NCOL; ++u)
                if (j0 + jj < nvalid) acc[u] = fma_rn(wj[jj], val[jj][u], acc[u]);
          }
        }
      }
      if (want_df && a.gfo_scalar) {
        const T val = a.gfo[0] * warp_sum(wsum);
        for (int cc = lane; cc < F; cc += 32) a.df[(int64_t)row * F + cc] = val;
      } else if (want_df) {
#pragma unroll
        for (int u = 0; u < NCOL; ++u) {
          const int cc = c0 + lane + 32 * u;
          if (cc < F) a.df[(int64_t)row * F + cc] = acc[u];
        }
      }
    }
    if (want_geo) {
      T vals[15];
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        vals[m] = gp[m];
        vals[3 + m] = gs[m];
      }
#pragma unroll
      for (int m = 0; m < 9; ++m) vals[6 + m] = gR[m];
#pragma unroll
      for (int m = 0; m < 15; ++m) vals[m] = warp_sum(vals[m]);
      if (lane == 0) {
        if (a.needs & KNNAG_NEED_DP)
          for (int m = 0; m < 3; ++m) a.dp[(int64_t)row * 3 + m] = vals[m];
        if (a.needs & KNNAG_NEED_DSIGMA)
          for (int m = 0; m < 3; ++m) a.dsigma[(int64_t)row * 3 + m] = vals[3 + m];
        if (a.needs & KNNAG_NEED_DR)
          for (int m = 0; m < 9; ++m) a.dR[(int64_t)row * 9 + m] = vals[6 + m];
      }
    }
  }
}

template <typename T, int ORDER, int NCOL>
__global__ void __launch_bounds__(256, 4) point_side_kernel(PointParams<T> a) {
  point_side_body<T, ORDER, NCOL>(a, blockIdx.x, gridDim.x);
}

// The second-order query side and point side in one launch: they read the
// same inputs (ggq, coef, records) and write disjoint outputs, so the first
// q_blocks CTAs run the query side and the rest the point side, side by side
// instead of one after the other.
template <typename T, int NCOL>
__global__ void __launch_bounds__(256, 3) order2_fused_kernel(QueryParams<T> qa, PointParams<T> pa, int q_blocks) {
  if ((int)blockIdx.x < q_blocks)
    query_order2_body(qa, blockIdx.x, q_blocks);
  else
    point_side_body<T, 2, NCOL>(pa, blockIdx.x - q_blocks, gridDim.x - q_blocks);
}

// ------------------------------------------------------------------ host

BwdLayout bwd_layout(int B, int Q, int P, int F, int K, int dtype) {
  BwdLayout L{};
  const size_t esz = dtype == KNNAG_F64 ? 8 : 4;
  size_t off = 0;
  L.status = off;
  off += 256;
  L.rec = off;
  off += align256((size_t)B * P * kRecLen * esz);
  L.adj = off;
  off += adj_layout(B, Q, P, K).total;
  L.coef = off;
  off += align256((size_t)B * Q * K * esz);
  L.rowsum = off;
  off += align256((size_t)B * P * esz);
  L.total = off;
  return L;
}

namespace {

template <typename T>
int launch_query(const QueryParams<T>& p, int order, cudaStream_t st) {
  NvtxRange range("knnag:query_side");
  const int64_t warps = (int64_t)p.B * p.Q;
  const unsigned grid = blocks_for(warps * 32, 256);
  if (order == 1)
    query_order1_kernel<T><<<grid, 256, 0, st>>>(p);
  else
    query_order2_kernel<T><<<grid, 256, 0, st>>>(p);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

}  // namespace

// d(<gfo, f_out>)/dq of a ragged call (gfo null: all ones), weights
// recomputed from idxs.  One warp per query row up to the table's total.
int ragged_grad_q_impl(const char* cs, const void* segs, const float* q, const float* f, int F, const float* gfo,
                       const float* f_row_sums, const int64_t* idxs, int64_t cap_q, float* dq, const int* status,
                       cudaStream_t st) {
  QueryParams<float> p{};
  p.status = status;
  if (!gfo) p.frowsum = f_row_sums;  // all-ones grad_f_out: c = rowsum(f)[idx]
  p.gfo = gfo;
  p.q = q;
  p.f = f;
  p.idxs = idxs;
  p.F = F;
  p.dq = dq;
  p.cs = cs;
  p.segs = segs;
  query_order1_kernel<float><<<blocks_for(cap_q * 32, 256), 256, 0, st>>>(p);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

int launch_row_sums(const void* f, int64_t rows, int F, int dtype, void* out, cudaStream_t st) {
  if (dtype == KNNAG_F64)
    row_sum_kernel<double><<<blocks_for(rows * 32, 256), 256, 0, st>>>((const double*)f, rows, F, (double*)out);
  else
    row_sum_kernel<float><<<blocks_for(rows * 32, 256), 256, 0, st>>>((const float*)f, rows, F, (float*)out);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

namespace {

template <typename T, int ORDER>
int launch_point_o(const PointParams<T>& p, cudaStream_t st) {
  const int64_t rows = (int64_t)p.B * p.P;
  const unsigned grid = blocks_for(rows * 32, 256);
  if (p.F <= 32)
    point_side_kernel<T, ORDER, 1><<<grid, 256, 0, st>>>(p);
  else if (p.F <= 64)
    point_side_kernel<T, ORDER, 2><<<grid, 256, 0, st>>>(p);
  else if (p.F <= 128)
    point_side_kernel<T, ORDER, 4><<<grid, 256, 0, st>>>(p);
  else
    point_side_kernel<T, ORDER, 8><<<grid, 256, 0, st>>>(p);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template <typename T>
int launch_order2_fused(const QueryParams<T>& qa, const PointParams<T>& pa, cudaStream_t st) {
  const unsigned qb = blocks_for((int64_t)qa.B * qa.Q * 32, 256);
  const unsigned pb = blocks_for((int64_t)pa.B * pa.P * 32, 256);
  const unsigned grid = qb + pb;
  if (pa.F <= 32)
    order2_fused_kernel<T, 1><<<grid, 256, 0, st>>>(qa, pa, (int)qb);
  else if (pa.F <= 64)
    order2_fused_kernel<T, 2><<<grid, 256, 0, st>>>(qa, pa, (int)qb);
  else if (pa.F <= 128)
    order2_fused_kernel<T, 4><<<grid, 256, 0, st>>>(qa, pa, (int)qb);
  else
    order2_fused_kernel<T, 8><<<grid, 256, 0, st>>>(qa, pa, (int)qb);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

template <typename T>
int backward_t(const BwdArgs& x, cudaStream_t st) {
  NvtxRange range(x.order == 1 ? "knnag:backward" : "knnag:backward_2nd");
  const BwdLayout L = bwd_layout(x.B, x.Q, x.P, x.F, x.K, x.dtype);
  char* ws = static_cast<char*>(x.workspace);
  int rc = KNNAG_OK;
  if (cudaMemsetAsync(ws + L.status, 0, 8, st) != cudaSuccess) return KNNAG_ERR_CUDA;
  const void* rec = x.points;
  if (!rec) {
    rc = launch_pack_points(x.p, x.sigma, x.R, x.B, x.P, x.dtype, ws + L.rec, st);
    if (rc) return rc;
    rec = ws + L.rec;
  }
  const int point_bits = KNNAG_NEED_DP | KNNAG_NEED_DF | KNNAG_NEED_DSIGMA | KNNAG_NEED_DR;
  const int geo_bits = KNNAG_NEED_DP | KNNAG_NEED_DSIGMA | KNNAG_NEED_DR;

  const T* coef = static_cast<const T*>(x.coef_in);
  const bool need_coef = (x.order == 1) ? (x.needs & geo_bits) != 0
                                         : (x.needs & (geo_bits | KNNAG_NEED_DQ)) != 0;
  T* coef_ws = reinterpret_cast<T*>(ws + L.coef);
  T* coef_out = static_cast<T*>(x.coef_out);

  const bool gfo_scalar = (x.needs & KNNAG_GFO_SCALAR) != 0;
  T* rowsum = reinterpret_cast<T*>(ws + L.rowsum);
  bool rowsum_ready = false;
  bool query2_pending = false;
  // per-point column sums of f, for the query side with a broadcast grad_f_out
  auto ensure_rowsum = [&]() -> int {
    if (rowsum_ready) return KNNAG_OK;
    row_sum_kernel<T><<<blocks_for((int64_t)x.B * x.P * 32, 256), 256, 0, st>>>((const T*)x.f, (int64_t)x.B * x.P,
                                                                                  x.F, rowsum);
    note_launches(1);
    rowsum_ready = true;
    return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
  };

  QueryParams<T> qp{};
  qp.gfo = (const T*)x.gfo;
  qp.ggq = (const T*)x.ggq;
  qp.q = (const T*)x.q;
  qp.rec = (const T*)rec;
  qp.f = (const T*)x.f;
  qp.w_in = (const T*)x.w_in;
  qp.idxs = x.idxs;
  qp.B = x.B;
  qp.Q = x.Q;
  qp.P = x.P;
  qp.F = x.F;
  qp.K = x.K;

  if (x.order == 1) {
    T* cdst = coef_out ? coef_out : (need_coef ? coef_ws : nullptr);
    if ((x.needs & KNNAG_NEED_DQ) || cdst) {
      qp.dq = (x.needs & KNNAG_NEED_DQ) ? (T*)x.dq : nullptr;
      qp.coef_out = cdst;
      if (gfo_scalar) {
        if ((rc = ensure_rowsum())) return rc;
        qp.frowsum = rowsum;
      }
      rc = launch_query<T>(qp, 1, st);
      if (rc) return rc;
    }
    coef = cdst;
  } else {
    if (!coef && need_coef) {
      QueryParams<T> cp = qp;
      cp.dq = nullptr;
      cp.coef_out = coef_ws;
      if (gfo_scalar) {
        if ((rc = ensure_rowsum())) return rc;
        cp.frowsum = rowsum;
      }
      rc = launch_query<T>(cp, 1, st);
      if (rc) return rc;
      coef = coef_ws;
    }
    if (x.needs & (KNNAG_NEED_DQ | KNNAG_NEED_DGFO)) {
      qp.coef_in = coef;
      qp.dq = (x.needs & KNNAG_NEED_DQ) ? (T*)x.dq : nullptr;
      qp.dgfo = (x.needs & KNNAG_NEED_DGFO) ? (T*)x.dgfo : nullptr;
      query2_pending = true;  // launched with the point side when that runs too
    }
  }

  if (x.needs & point_bits) {
    NvtxRange r("knnag:point_side");
    const void* adj = x.adjacency;
    if (!adj) {
      rc = launch_build_adjacency(x.idxs, x.B, x.Q, x.P, x.K, ws + L.adj, st);
      if (rc) return rc;
      adj = ws + L.adj;
    }
    const AdjLayout AL = adj_layout(x.B, x.Q, x.P, x.K);
    PointParams<T> pp{};
    pp.gfo = (const T*)x.gfo;
    pp.ggq = (const T*)x.ggq;
    pp.q = (const T*)x.q;
    pp.rec = (const T*)rec;
    pp.w_in = (const T*)x.w_in;
    pp.coef = coef;
    pp.rowptr = reinterpret_cast<const int*>(static_cast<const char*>(adj) + AL.rowptr);
    pp.entries = reinterpret_cast<const int*>(static_cast<const char*>(adj) + AL.entries);
    pp.B = x.B;
    pp.Q = x.Q;
    pp.P = x.P;
    pp.F = x.F;
    pp.K = x.K;
    pp.needs = x.needs;
    pp.dp = (T*)x.dp;
    pp.df = (T*)x.df;
    pp.dsigma = (T*)x.dsigma;
    pp.dR = (T*)x.dR;
    pp.gfo_scalar = gfo_scalar;
    if (query2_pending && sizeof(T) == 4) {  // FP64 keeps separate launches (the fused one spills)
      NvtxRange r2("knnag:query_side");
      return launch_order2_fused<T>(qp, pp, st);
    }
    if (query2_pending && (rc = launch_query<T>(qp, 2, st))) return rc;
    rc = (x.order == 1) ? launch_point_o<T, 1>(pp, st) : launch_point_o<T, 2>(pp, st);
    return rc;
  }
  if (query2_pending) rc = launch_query<T>(qp, 2, st);
  return rc;
}

}  // namespace

int backward_impl(const BwdArgs& x, cudaStream_t st) {
  return x.dtype == KNNAG_F64 ? backward_t<double>(x, st) : backward_t<float>(x, st);
}

}  // namespace knnag
