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

__global__ void adj_count_kernel(const int64_t* __restrict__ idxs, int64_t n, int64_t qk, int P,
                                 int* __restrict__ count) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = e / qk;
    const int64_t idx = idxs[e];
    if (idx < 0 || idx >= P) continue;  // not a point index: no row holds it
    atomicAdd(&count[b * P + idx], 1);
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

__global__ void adj_fill_kernel(const int64_t* __restrict__ idxs, int64_t n, int64_t qk, int P,
                                const int* __restrict__ rowptr, int* __restrict__ cursor, int* __restrict__ unsorted) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t idx = idxs[e];
    if (idx < 0 || idx >= P) continue;
    const int64_t row = (e / qk) * P + idx;
    const int pos = rowptr[row] + atomicAdd(&cursor[row], 1);
    unsorted[pos] = (int)e;
  }
}

// Sort every row by entry id: one warp per row; an entry's slot is the
// number of smaller ids in its row (ids in a row are distinct because a
// query selects a point at most once; equal ids keep their order).
__global__ void adj_sort_kernel(const int* __restrict__ rowptr, const int* __restrict__ unsorted, int64_t n_rows,
                                int* __restrict__ entries) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = gw; r < n_rows; r += nw) {
    const int start = rowptr[r];
    const int n = rowptr[r + 1] - start;
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const int v = (i < n) ? unsorted[start + i] : 0;
      int rank = 0;
      for (int jb = 0; jb < n; jb += 32) {
        const int uj = (jb + lane < n) ? unsorted[start + jb + lane] : 0x7fffffff;
        const int lim = min(32, n - jb);
        for (int jj = 0; jj < lim; ++jj) {
          const int u = __shfl_sync(0xffffffffu, uj, jj);
          rank += (u < v || (u == v && jb + jj < i)) ? 1 : 0;  // stable even if ids repeat
        }
      }
      if (i < n) entries[start + rank] = v;
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

int launch_build_adjacency(const int64_t* idxs, int B, int Q, int P, int K, void* adjacency, cudaStream_t st) {
  const AdjLayout L = adj_layout(B, Q, P, K);
  char* base = static_cast<char*>(adjacency);
  int* rowptr = reinterpret_cast<int*>(base + L.rowptr);
  int* cursor = reinterpret_cast<int*>(base + L.cursor);
  int* unsorted = reinterpret_cast<int*>(base + L.unsorted);
  int* entries = reinterpret_cast<int*>(base + L.entries);
  const int64_t n = (int64_t)B * Q * K, rows = (int64_t)B * P, qk = (int64_t)Q * K;
  if (cudaMemsetAsync(cursor, 0, (size_t)rows * 4, st) != cudaSuccess) return KNNAG_ERR_CUDA;
  adj_count_kernel<<<blocks_for(n, 256), 256, 0, st>>>(idxs, n, qk, P, cursor);
  adj_scan_kernel<<<1, 1024, 0, st>>>(cursor, rows, rowptr);
  adj_fill_kernel<<<blocks_for(n, 256), 256, 0, st>>>(idxs, n, qk, P, rowptr, cursor, unsorted);
  adj_sort_kernel<<<blocks_for(rows * 32, 256), 256, 0, st>>>(rowptr, unsorted, rows, entries);
  note_launches(4);
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
};

// v = R^T diag(sigma) u
template <typename T>
__device__ __forceinline__ void rot_back(const T* r, const T* sg, const T* u, T* v) {
#pragma unroll
  for (int m = 0; m < 3; ++m) v[m] = sg[0] * u[0] * r[m] + sg[1] * u[1] * r[3 + m] + sg[2] * u[2] * r[6 + m];
}

// Half-warp (16 lanes) per query: dot products c_k = gfo[q] . f[idx_k] are
// split over the 16 lanes (128-bit loads when V4) and tree-reduced; the
// geometry of entry k0+l is done by lane l of the half-warp.
template <typename T, int ORDER, bool V4>
__global__ void __launch_bounds__(128) query_side_kernel(QueryParams<T> a) {
  const int hl = threadIdx.x & 15;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int64_t BQ = (int64_t)a.B * a.Q;
  const int K = a.K, F = a.F, P = a.P;
  const bool need_dot = (ORDER == 1) || a.coef_in == nullptr;
  for (int64_t bq = blockIdx.x * 8 + (threadIdx.x >> 4); bq < BQ; bq += (int64_t)gridDim.x * 8) {
    const int64_t b = bq / a.Q;
    const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];
    T g[3] = {T(0), T(0), T(0)};
    if (ORDER == 2) {
      g[0] = a.ggq[bq * 3 + 0];
      g[1] = a.ggq[bq * 3 + 1];
      g[2] = a.ggq[bq * 3 + 2];
    }
    const T* grow = a.gfo + bq * F;
    const T* fb = a.f + b * (int64_t)P * F;
    T acc[3] = {T(0), T(0), T(0)};
    for (int k0 = 0; k0 < K; k0 += 16) {
      const int nk = min(16, K - k0);
      T c_own = T(0);
      if (need_dot) {
        for (int kk = 0; kk < nk; ++kk) {
          const int64_t idx = a.idxs[bq * K + k0 + kk];
          const T* frow = fb + idx * F;
          T part = T(0);
          if (idx < 0 || idx >= P) {
            // not a point index: contributes nothing
          } else if (V4) {
            const float4* g4 = reinterpret_cast<const float4*>(grow);
            const float4* f4 = reinterpret_cast<const float4*>(frow);
            for (int c = hl; c < (F >> 2); c += 16) {
              const float4 x = __ldg(g4 + c), y = __ldg(f4 + c);
              part = fma_rn((T)x.x, (T)y.x, part);
              part = fma_rn((T)x.y, (T)y.y, part);
              part = fma_rn((T)x.z, (T)y.z, part);
              part = fma_rn((T)x.w, (T)y.w, part);
            }
          } else {
            for (int c = hl; c < F; c += 16) part = fma_rn(grow[c], frow[c], part);
          }
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(hmask, part, o, 16);
          if (hl == kk) c_own = part;
        }
      } else if (hl < nk) {
        c_own = a.coef_in[bq * K + k0 + hl];
      }
      T a_own = T(0);
      const int64_t e_own = bq * K + k0 + hl;
      const int64_t i_own = (hl < nk) ? a.idxs[e_own] : -1;
      if (hl < nk && a.coef_out) a.coef_out[e_own] = c_own;
      if (i_own >= 0 && i_own < P) {
        const int64_t e = e_own;
        const T* rec = a.rec + (b * P + i_own) * kRecLen;
        Geo<T> geo;
        geometry(qx, qy, qz, rec, geo);
        const T w = a.w_in ? a.w_in[e] : geo.w;
        const T* r = rec + kR00;
        const T sg[3] = {rec[kS0], rec[kS1], rec[kS2]};
        T v[3];
        rot_back(r, sg, geo.u, v);
        if (ORDER == 1) {
          const T t = T(-2) * c_own * w;
#pragma unroll
          for (int m = 0; m < 3; ++m) acc[m] += t * v[m];
        } else {
          const T A = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
          T rg[3];
#pragma unroll
          for (int s = 0; s < 3; ++s) rg[s] = r[3 * s] * g[0] + r[3 * s + 1] * g[1] + r[3 * s + 2] * g[2];
          const T cw2 = T(2) * c_own * w;
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const T mg = sg[0] * rg[0] * r[m] + sg[1] * rg[1] * r[3 + m] + sg[2] * rg[2] * r[6 + m];
            acc[m] += cw2 * (T(2) * A * v[m] - mg);
          }
          a_own = T(-2) * w * A;
        }
      }
      if (ORDER == 2 && a.dgfo) {
        T ak[16];
        int64_t ik[16];
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
          ak[kk] = __shfl_sync(hmask, a_own, kk, 16);
          ik[kk] = (kk < nk) ? a.idxs[bq * K + k0 + kk] : -1;
          if (ik[kk] >= P) ik[kk] = -1;
        }
        T* drow = a.dgfo + bq * F;
        for (int c = hl; c < F; c += 16) {
          T s = (k0 == 0) ? T(0) : drow[c];
#pragma unroll
          for (int kk = 0; kk < 16; ++kk)
            if (kk < nk && ik[kk] >= 0) s = fma_rn(ak[kk], fb[ik[kk] * F + c], s);
          drow[c] = s;
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) acc[m] += __shfl_xor_sync(hmask, acc[m], o, 16);
    }
    if (hl == 0 && a.dq) {
      a.dq[bq * 3 + 0] = acc[0];
      a.dq[bq * 3 + 1] = acc[1];
      a.dq[bq * 3 + 2] = acc[2];
    }
  }
}

// One warp per point row.  Lane j takes entry j of each 32-entry chunk of
// the row for the per-entry geometry (15 point-side scalars, reduced over
// the warp at the end); for df the warp then walks the chunk entry by entry
// with lanes spanning feature columns (NCOL per lane, coalesced gfo rows).
template <typename T, int ORDER, int NCOL>
__global__ void __launch_bounds__(256) point_side_kernel(PointParams<T> a) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t rows = (int64_t)a.B * a.P;
  const int F = a.F, K = a.K;
  const bool want_geo = (a.needs & (KNNAG_NEED_DP | KNNAG_NEED_DSIGMA | KNNAG_NEED_DR)) != 0;
  const bool want_df = (a.needs & KNNAG_NEED_DF) != 0;
  for (int64_t row = gw; row < rows; row += nw) {
    const T* rec = a.rec + row * kRecLen;
    T pr[kRecLen];
#pragma unroll
    for (int m = 0; m < kRecLen; ++m) pr[m] = rec[m];
    const T* r = pr + kR00;
    const T sg[3] = {pr[kS0], pr[kS1], pr[kS2]};
    const int start = a.rowptr[row], end = a.rowptr[row + 1];
    T gp[3] = {T(0), T(0), T(0)}, gs[3] = {T(0), T(0), T(0)}, gR[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) gR[m] = T(0);
    for (int c0 = 0; c0 == 0 || (want_df && c0 < F); c0 += 32 * NCOL) {
      T acc[NCOL];
#pragma unroll
      for (int u = 0; u < NCOL; ++u) acc[u] = T(0);
      for (int base = start; base < end; base += 32) {
        const int j = base + lane;
        int64_t e = (j < end) ? (int64_t)a.entries[j] : -1;
        const bool valid = e >= 0 && e < (int64_t)a.B * a.Q * K;
        if (!valid) e = 0;
        const int64_t bq = e / K;
        T wgt = T(0);
        if (valid) {
          const T qx = a.q[bq * 3 + 0], qy = a.q[bq * 3 + 1], qz = a.q[bq * 3 + 2];
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
              for (int s = 0; s < 3; ++s) {
                gs[s] -= cw * geo.u[s] * geo.u[s];
                const T t = T(-2) * cw * sg[s] * geo.u[s];
#pragma unroll
                for (int m = 0; m < 3; ++m) gR[3 * s + m] += t * geo.d[m];
              }
            }
          } else {
            const T g[3] = {a.ggq[bq * 3 + 0], a.ggq[bq * 3 + 1], a.ggq[bq * 3 + 2]};
            const T A = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
            wgt = T(-2) * w * A;
            if (want_geo && c0 == 0) {
              T rg[3];
#pragma unroll
              for (int s = 0; s < 3; ++s) rg[s] = r[3 * s] * g[0] + r[3 * s + 1] * g[1] + r[3 * s + 2] * g[2];
              const T cw = c * w;
#pragma unroll
              for (int m = 0; m < 3; ++m) {
                const T mg = sg[0] * rg[0] * r[m] + sg[1] * rg[1] * r[3 + m] + sg[2] * rg[2] * r[6 + m];
                gp[m] -= T(2) * cw * (T(2) * A * v[m] - mg);
              }
#pragma unroll
              for (int s = 0; s < 3; ++s) {
                gs[s] += T(2) * cw * geo.u[s] * (geo.u[s] * A - rg[s]);
                const T t = T(-2) * cw * sg[s];
#pragma unroll
                for (int m = 0; m < 3; ++m)
                  gR[3 * s + m] += t * (T(-2) * geo.u[s] * geo.d[m] * A + geo.d[m] * rg[s] + geo.u[s] * g[m]);
              }
            }
          }
        }
        if (want_df) {
          const int nvalid = min(32, end - base);
          for (int jj = 0; jj < nvalid; ++jj) {
            const int64_t bqj = __shfl_sync(0xffffffffu, bq, jj);
            const T wj = __shfl_sync(0xffffffffu, wgt, jj);
            const T* grow = a.gfo + bqj * F;
#pragma unroll
            for (int u = 0; u < NCOL; ++u) {
              const int c = c0 + lane + 32 * u;
              if (c < F) acc[u] = fma_rn(wj, grow[c], acc[u]);
            }
          }
        }
      }
      if (want_df) {
#pragma unroll
        for (int u = 0; u < NCOL; ++u) {
          const int c = c0 + lane + 32 * u;
          if (c < F) a.df[row * F + c] = acc[u];
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
      for (int m = 0; m < 15; ++m) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vals[m] += __shfl_xor_sync(0xffffffffu, vals[m], o);
      }
      if (lane == 0) {
        if (a.needs & KNNAG_NEED_DP)
          for (int m = 0; m < 3; ++m) a.dp[row * 3 + m] = vals[m];
        if (a.needs & KNNAG_NEED_DSIGMA)
          for (int m = 0; m < 3; ++m) a.dsigma[row * 3 + m] = vals[3 + m];
        if (a.needs & KNNAG_NEED_DR)
          for (int m = 0; m < 9; ++m) a.dR[row * 9 + m] = vals[6 + m];
      }
    }
  }
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
  L.total = off;
  return L;
}

namespace {

template <typename T>
int launch_query(const QueryParams<T>& p, int order, bool v4, cudaStream_t st) {
  const int64_t bq = (int64_t)p.B * p.Q;
  const unsigned grid = blocks_for(bq * 16, 128);
  if (order == 1) {
    if (v4)
      query_side_kernel<T, 1, true><<<grid, 128, 0, st>>>(p);
    else
      query_side_kernel<T, 1, false><<<grid, 128, 0, st>>>(p);
  } else {
    if (v4)
      query_side_kernel<T, 2, true><<<grid, 128, 0, st>>>(p);
    else
      query_side_kernel<T, 2, false><<<grid, 128, 0, st>>>(p);
  }
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

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
int backward_t(const BwdArgs& x, cudaStream_t st) {
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
  const bool v4 = sizeof(T) == 4 && x.F % 4 == 0 && (uintptr_t)x.gfo % 16 == 0 && (uintptr_t)x.f % 16 == 0;

  const T* coef = static_cast<const T*>(x.coef_in);
  const bool need_coef = (x.order == 1) ? (x.needs & geo_bits) != 0
                                         : (x.needs & (geo_bits | KNNAG_NEED_DQ)) != 0;
  T* coef_ws = reinterpret_cast<T*>(ws + L.coef);
  T* coef_out = static_cast<T*>(x.coef_out);

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
      rc = launch_query<T>(qp, 1, v4, st);
      if (rc) return rc;
    }
    coef = cdst;
  } else {
    if (!coef && need_coef) {
      QueryParams<T> cp = qp;
      cp.dq = nullptr;
      cp.coef_out = coef_ws;
      rc = launch_query<T>(cp, 1, v4, st);
      if (rc) return rc;
      coef = coef_ws;
    }
    if (x.needs & (KNNAG_NEED_DQ | KNNAG_NEED_DGFO)) {
      qp.coef_in = coef;
      qp.dq = (x.needs & KNNAG_NEED_DQ) ? (T*)x.dq : nullptr;
      qp.dgfo = (x.needs & KNNAG_NEED_DGFO) ? (T*)x.dgfo : nullptr;
      rc = launch_query<T>(qp, 2, v4, st);
      if (rc) return rc;
    }
  }

  if (x.needs & point_bits) {
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
    rc = (x.order == 1) ? launch_point_o<T, 1>(pp, st) : launch_point_o<T, 2>(pp, st);
  }
  return rc;
}

}  // namespace

int backward_impl(const BwdArgs& x, cudaStream_t st) {
  return x.dtype == KNNAG_F64 ? backward_t<double>(x, st) : backward_t<float>(x, st);
}

}  // namespace knnag
