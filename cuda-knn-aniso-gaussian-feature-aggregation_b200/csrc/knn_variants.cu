// The reference's other forward ops:
//   * aggregation at caller-given neighbour indices
//     (knn_precomputed_aggregate_aniso_forward, csrc/forward.cu:186-230);
//   * the lookup variant: Euclidean nearest point, then its row of a
//     neighbour table (knn_lookup_aggregate_aniso_forward,
//     csrc/forward.cu:113-183);
//   * the isotropic forward (knn_aggregate_forward, csrc/forward.cu:5-53),
//     served by the exact MinK kernel with Euclidean keys.
// Keys, weights and sums use the same arithmetic and order as the reference,
// so dists / w_out / f_out match it bit for bit.
#include <math.h>

#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {

// One warp per query.  Lane k (and k+32, ...) takes neighbour k: key from the
// packed record, w = exp(-key) (-> dists, w_out); the warp then sums
// f_out = sum_k w_k f[idx_k] in k order with lanes spanning columns.  The
// neighbour index comes from `idxs` [B,Q,K] or, for the lookup, from
// `table` [P,K] at row nearest[b*Q+q] (and is written to idxs_out).  An
// index outside [0, P) contributes nothing (w = 0, dist = +inf).
template <typename T>
__global__ void __launch_bounds__(256) gather_aggregate_kernel(const T* __restrict__ q, const T* __restrict__ f,
                                                              const T* __restrict__ rec,
                                                              const int64_t* __restrict__ idxs,
                                                              const int64_t* __restrict__ table,
                                                              const int* __restrict__ nearest, int tstride, int B,
                                                              int Q, int P, int F, int K, T* __restrict__ f_out,
                                                              T* __restrict__ w_out, T* __restrict__ dists,
                                                              int64_t* __restrict__ idxs_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* sw = reinterpret_cast<T*>(smem_raw) + (size_t)warp * K;
  int* si = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + (size_t)8 * K) + (size_t)warp * K;
  const int BQ = B * Q;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int bq = gw; bq < BQ; bq += nw) {
    const int b = bq / Q;
    const T qx = q[(int64_t)bq * 3 + 0], qy = q[(int64_t)bq * 3 + 1], qz = q[(int64_t)bq * 3 + 2];
    const int64_t row = table ? (int64_t)nearest[bq] : 0;
    for (int k = lane; k < K; k += 32) {
      const int64_t e = (int64_t)bq * K + k;
      const int64_t idx = table ? table[row * tstride + k] : idxs[e];
      T key = T(INFINITY), w = T(0);
      if (idx >= 0 && idx < P) {
        key = key_rec<T>(qx, qy, qz, rec + ((int64_t)b * P + idx) * kRecLen);
        w = weight_of(key);
      }
      dists[e] = key;
      w_out[e] = w;
      if (idxs_out) idxs_out[e] = idx;
      sw[k] = w;
      si[k] = (idx >= 0 && idx < P) ? (int)idx : -1;
    }
    __syncwarp();
    const T* fb = f + (int64_t)b * P * F;
    for (int c0 = 0; c0 < F; c0 += 32) {
      const int c = c0 + lane;
      if (c < F) {
        T acc = T(0);
        for (int k = 0; k < K; ++k)
          if (si[k] >= 0) acc = fma_rn(fb[(int64_t)si[k] * F + c], sw[k], acc);
        f_out[(int64_t)bq * F + c] = acc;
      }
    }
    __syncwarp();
  }
}

// Euclidean nearest point of every query: strict '<' scan in index order
// from 1e10 (the first index wins ties; 0 when no distance is below 1e10),
// d = fma(z,z, fma(x,x, y*y)) for x*x + y*y + z*z (csrc/forward.cu:141-160).
// One thread per query, 256 queries per CTA, points staged 1024 at a time.
template <typename T>
__global__ void __launch_bounds__(256) nearest_point_kernel(const T* __restrict__ q, const T* __restrict__ p, int B,
                                                           int Q, int P, int* __restrict__ nearest) {
  constexpr int CH = 1024;
  __shared__ T sp[CH * 3];
  const int b = blockIdx.y;
  const int qi = blockIdx.x * 256 + threadIdx.x;
  const bool valid = qi < Q;
  const int64_t bq = (int64_t)b * Q + (valid ? qi : 0);
  const T qx = q[bq * 3 + 0], qy = q[bq * 3 + 1], qz = q[bq * 3 + 2];
  T best = T(1e10);
  int arg = 0;
  const T* pb = p + (int64_t)b * P * 3;
  for (int c0 = 0; c0 < P; c0 += CH) {
    const int n = min(CH, P - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < n * 3; i += 256) sp[i] = pb[(int64_t)c0 * 3 + i];
    __syncthreads();
    for (int i = 0; i < n; ++i) {
      const T x = qx - sp[3 * i], y = qy - sp[3 * i + 1], z = qz - sp[3 * i + 2];
      const T d = fma_rn(z, z, fma_rn(x, x, mul_rn(y, y)));
      if (d < best) {
        best = d;
        arg = c0 + i;
      }
    }
  }
  if (valid) nearest[bq] = arg;
}

namespace {
int variant_blocks(int64_t warps) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t b = (warps * 32 + 255) / 256;
  const int64_t cap = (int64_t)sms * 16;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
int launch_gather(const T* q, const T* f, const T* rec, const int64_t* idxs, const int64_t* table, const int* nearest,
                  int tstride, int B, int Q, int P, int F, int K, T* f_out, T* w_out, T* dists, int64_t* idxs_out,
                  cudaStream_t st) {
  const size_t smem = (size_t)8 * K * (sizeof(T) + sizeof(int));
  if (smem > 200 * 1024) return KNNAG_ERR_TOO_LARGE;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(gather_aggregate_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return KNNAG_ERR_CUDA;
  gather_aggregate_kernel<T><<<variant_blocks((int64_t)B * Q), 256, smem, st>>>(q, f, rec, idxs, table, nearest, tstride,
                                                                                 B, Q, P, F, K, f_out, w_out, dists,
                                                                                 idxs_out);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}
}  // namespace

int variants_precomputed(const void* q, const void* f, const void* rec, const int64_t* idxs, int B, int Q, int P,
                         int F, int K, int dtype, void* f_out, void* w_out, void* dists, cudaStream_t st) {
  if (dtype == KNNAG_F64)
    return launch_gather<double>((const double*)q, (const double*)f, (const double*)rec, idxs, nullptr, nullptr, K, B,
                                 Q, P, F, K, (double*)f_out, (double*)w_out, (double*)dists, nullptr, st);
  return launch_gather<float>((const float*)q, (const float*)f, (const float*)rec, idxs, nullptr, nullptr, K, B, Q, P,
                              F, K, (float*)f_out, (float*)w_out, (float*)dists, nullptr, st);
}

int variants_lookup(const void* q, const void* p, const void* f, const void* rec, const int64_t* table, int tstride, int B, int Q,
                    int P, int F, int K, int dtype, int* nearest, void* f_out, void* w_out, void* dists,
                    int64_t* idxs, cudaStream_t st) {
  dim3 grid((Q + 255) / 256, B);
  if (dtype == KNNAG_F64)
    nearest_point_kernel<double><<<grid, 256, 0, st>>>((const double*)q, (const double*)p, B, Q, P, nearest);
  else
    nearest_point_kernel<float><<<grid, 256, 0, st>>>((const float*)q, (const float*)p, B, Q, P, nearest);
  note_launches(1);
  if (cudaGetLastError() != cudaSuccess) return KNNAG_ERR_CUDA;
  if (dtype == KNNAG_F64)
    return launch_gather<double>((const double*)q, (const double*)f, (const double*)rec, nullptr, table, nearest,
                                 tstride, B, Q, P, F, K, (double*)f_out, (double*)w_out, (double*)dists, idxs, st);
  return launch_gather<float>((const float*)q, (const float*)f, (const float*)rec, nullptr, table, nearest, tstride, B, Q,
                              P, F, K, (float*)f_out, (float*)w_out, (float*)dists, idxs, st);
}

}  // namespace knnag
