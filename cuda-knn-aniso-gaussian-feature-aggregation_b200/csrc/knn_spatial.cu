// Spatial ordering for the search: points and queries of every batch element
// are counting-sorted by the Hilbert-curve index of a uniform grid cell, the search
// tiles are packed in that order (each record keeps its original point
// index), and every 128-point tile gets an axis-aligned box and a lower bound
// on the key of any query against any of its points:
//     key(q, i) >= mu_tile * dist(q, box_tile)^2,
//     mu_tile = min over the tile's points of  lambda_min(R^T diag(sigma) R)
//               - 1e-5 * sum_a |sigma_a| |R_a|^2,
// where lambda_min is computed in double and the second term covers the
// rounding of the FP32 key (|key_fp32 - key_exact| <= ~12 * 2^-24 *
// |q - p|^2 * sum_a |sigma_a| |R_a|^2).  With every sigma >= 0 every key is
// >= 0, so mu = 0 still bounds; a tile holding a negative or non-finite
// value gets mu = -1: no bound at all (its keys may be negative).
// The search visits tiles nearest-first by this bound and stops when the
// bound exceeds every query's threshold; the order of points inside a cell
// (atomic scatter) never changes a result, only the work done.
#include <math.h>

#include <algorithm>

#include "knn_common.cuh"
#include "knn_internal.h"

namespace knnag {

// Element groups of a counting sort: the batch elements of a uniform batch
// (group g = elements [g*n, (g+1)*n), cells [g*8^bits, ...)), the clouds of
// a cloud set, or the segments of a segment table (whose bounds are their
// cloud's).  Positions of group g in the sorted order start where its first
// element does, because the scan runs over [group][cell].
struct GroupRange {
  int64_t start;
  int n, cell_off, bits, bnd;
};
struct GroupMap {
  int n, bits;               // uniform batches
  const CloudDesc* clouds;   // cloud set (points)
  const SegDesc* segs;       // segment table (queries)
  const SegHeader* seg_hdr;  // live segment count
  const char* cs;            // cloud set whose bounds the segments use
  const int* status;         // segments: nothing is done once this is nonzero
};
// Bounds array of a map: the cloud set's own for segments, else `bnd`.
__device__ __forceinline__ const float* group_bounds(const GroupMap& m, const float* bnd) {
  return m.cs ? reinterpret_cast<const float*>(m.cs + reinterpret_cast<const CloudSetHeader*>(m.cs)->bnd_off) : bnd;
}
__device__ __forceinline__ bool group_range(const GroupMap& m, int g, GroupRange& r) {
  if (m.segs) {
    if ((m.status && *m.status) || g >= m.seg_hdr->nseg) return false;
    const SegDesc& s = m.segs[g];
    r = GroupRange{s.q_off, s.Q, s.qcell_off, s.qbits, s.cloud};
  } else if (m.clouds) {
    const CloudDesc& c = m.clouds[g];
    r = GroupRange{c.p_off, c.P, c.cell_off, c.bits, g};
  } else {
    r = GroupRange{(int64_t)g * m.n, m.n, g << (3 * m.bits), m.bits, g};
  }
  return true;
}

// Per group of points: bounding box, bnd[g] = {min xyz, max xyz}.
__global__ void __launch_bounds__(512) point_bounds_kernel(const float* __restrict__ rec, GroupMap m,
                                                           float* __restrict__ bnd) {
  __shared__ float red[6][16];
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  GroupRange r;
  group_range(m, b, r);
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll 4
  for (int i = tid; i < r.n; i += blockDim.x) {
    const float* rr = rec + (r.start + i) * kRecLen;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = -rr[kNPX + a];
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
    bnd[b * 8 + tid] = v;
  }
}

// A counting-sort job: the elements of the groups of `m` (points from
// records, or queries from q) and where their cells start in the shared
// count / offset arrays.  One launch can run two jobs (blockIdx.z), e.g. the
// points and the queries of a batch, whose cells are then scanned together.
struct CellJob {
  const float* xyz;
  int stride, negate;
  GroupMap m;
  int cell_base;
  int nparts;  // > 0: bnd holds nparts partial boxes per group, reduced here
  // queries of a uniform batch sorted together with its points (whose cells
  // come first in the scan): seed[position - seed_sub] = the middle of the
  // element's cell in its group's sorted points
  int* seed;
  int64_t seed_sub;
};

// Seed position of an element in cell c (global index in the scanned
// arrays) of the query job j: the middle of the same cell's points, as a
// position in the group's sorted points.  The points' cells of group r sit
// at r.cell_off + (c - j.cell_base); off[] is the exclusive scan.
__device__ __forceinline__ int seed_of(const CellJob& j, const GroupRange& r, const int* off, int c) {
  const int pc = c - j.cell_base;
  return ((off[pc] + off[pc + 1]) >> 1) - off[r.cell_off];
}

// The box of group r: bnd's entry, or the reduction of its nparts partial
// boxes (into shared memory, by the first threads of the CTA; all threads
// of the CTA must call this).
__device__ __forceinline__ const float* job_bounds(const CellJob& j, const float* bnd, const GroupRange& r,
                                                   float* gbs) {
  if (j.nparts <= 0) return group_bounds(j.m, bnd) + r.bnd * 8;
  if (threadIdx.x < 6) {
    const int a = threadIdx.x;
    float v = a < 3 ? INFINITY : -INFINITY;
    for (int i = 0; i < j.nparts; ++i) {
      const float x = bnd[((int64_t)r.bnd * j.nparts + i) * 8 + a];
      v = a < 3 ? fminf(v, x) : fmaxf(v, x);
    }
    gbs[a] = v;
  }
  __syncthreads();
  return gbs;
}

// Cell histogram of the elements of group blockIdx.y of job blockIdx.z.
__global__ void cell_count_kernel(CellJob j0, CellJob j1, const float* __restrict__ bnd, int* __restrict__ count) {
  __shared__ float gbs[6];
  const CellJob& j = blockIdx.z ? j1 : j0;
  GroupRange r;
  if (!group_range(j.m, blockIdx.y, r)) return;
  const float s = j.negate ? -1.f : 1.f;
  const float* gb = job_bounds(j, bnd, r, gbs);
  int* cnt = count + j.cell_base + r.cell_off;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
    const float* v = j.xyz + (r.start + i) * j.stride;
    atomicAdd(&cnt[cell_of(s * v[0], s * v[1], s * v[2], gb, r.bits)], 1);
  }
}

// perm[offset[cell] + rank] = index within the group.
__global__ void cell_scatter_kernel(CellJob j0, CellJob j1, const float* __restrict__ bnd,
                                    const int* __restrict__ offset, int* __restrict__ cursor, int* __restrict__ perm) {
  __shared__ float gbs[6];
  const CellJob& j = blockIdx.z ? j1 : j0;
  GroupRange r;
  if (!group_range(j.m, blockIdx.y, r)) return;
  const float s = j.negate ? -1.f : 1.f;
  const float* gb = job_bounds(j, bnd, r, gbs);
  const int base = j.cell_base + r.cell_off;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
    const float* v = j.xyz + (r.start + i) * j.stride;
    const int c = base + (int)cell_of(s * v[0], s * v[1], s * v[2], gb, r.bits);
    const int pos = offset[c] + atomicAdd(&cursor[c], 1);
    perm[pos] = i;
    if (j.seed) j.seed[pos - j.seed_sub] = seed_of(j, r, offset, c);
  }
}

// The scatter with the scan folded in, for at most kScatterScanMax cells:
// every CTA scans the cell counts into shared memory itself (a few KB
// read from L2), so no separate scan launch sits between the count and the
// scatter; `cursor` (zeroed beforehand) ranks the elements of a cell.
constexpr int kScatterScanMax = 8192;

__global__ void __launch_bounds__(256) cell_scatter_scan_kernel(CellJob j0, CellJob j1, const float* __restrict__ bnd,
                                                                const int* __restrict__ count, int nc,
                                                                int* __restrict__ cursor, int* __restrict__ perm) {
  __shared__ int soff[kScatterScanMax];
  __shared__ int wsum[8];
  __shared__ float gbs[6];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (nc + 255) / 256;  // <= 32 consecutive counts per thread
  int local = 0;
  for (int u = 0; u < per; ++u) {
    const int i = tid * per + u;
    if (i < nc) {
      const int v = count[i];
      soff[i] = v;
      local += v;
    }
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int run = incl - local;
  for (int w = 0; w < warp; ++w) run += wsum[w];
  for (int u = 0; u < per; ++u) {
    const int i = tid * per + u;
    if (i < nc) {
      const int v = soff[i];
      soff[i] = run;
      run += v;
    }
  }
  __syncthreads();
  const CellJob& j = blockIdx.z ? j1 : j0;
  GroupRange r;
  if (!group_range(j.m, blockIdx.y, r)) return;
  const float s = j.negate ? -1.f : 1.f;
  const float* gb = job_bounds(j, bnd, r, gbs);
  const int base = j.cell_base + r.cell_off;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
    const float* v = j.xyz + (r.start + i) * j.stride;
    const int c = base + (int)cell_of(s * v[0], s * v[1], s * v[2], gb, r.bits);
    const int pos = soff[c] + atomicAdd(&cursor[c], 1);
    perm[pos] = i;
    if (j.seed) j.seed[pos - j.seed_sub] = seed_of(j, r, soff, c);
  }
}

// Point groups of the tile kernels: uniform (group b: records [b*P, ...),
// tiles [b*ntile, ...)) or the clouds of a cloud set.
struct TileGroup {
  int64_t p0, t0;
  int P, ntile;
};
__device__ __forceinline__ TileGroup tile_group(const CloudDesc* cd, int b, int P, int ntile) {
  if (cd) return TileGroup{cd[b].p_off, cd[b].tile_off, cd[b].P, cd[b].ntile};
  return TileGroup{(int64_t)b * P, (int64_t)b * ntile, P, ntile};
}

// Smallest eigenvalue of a symmetric 3x3 matrix (closed form), double.
__device__ double sym3_min_eig(double a00, double a11, double a22, double a01, double a02, double a12) {
  const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
  if (p1 == 0.0) return fmin(a00, fmin(a11, a22));
  const double qm = (a00 + a11 + a22) / 3.0;
  const double b00 = a00 - qm, b11 = a11 - qm, b22 = a22 - qm;
  const double p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1;
  const double p = sqrt(p2 / 6.0);
  const double ip = 1.0 / p;
  const double c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = a01 * ip, c02 = a02 * ip, c12 = a12 * ip;
  double r = 0.5 * (c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02));
  r = fmin(1.0, fmax(-1.0, r));
  const double phi = acos(r) / 3.0;
  return qm + 2.0 * p * cos(phi + 2.0943951023931957);  // + 2 pi / 3
}

// Tensor-core filter operands of one tile, by the tile-info CTA (thread k:
// sorted point k, `real` unless padding; `tile` holds the records field-major,
// red[w][0..5] the box of warp w's points).  With o the tile's box centre,
// p' = p - o and M = R^T diag(sigma) R (in double), the point's features
//   psi = (M00, M11, M22, 2 M01, 2 M02, 2 M12, -2 (M p')_0..2, p'^T M p')
// meet a query's phi = (x^2, y^2, z^2, xy, xz, yz, x, y, z, 1), (x,y,z) =
// q - o, in phi . psi = (q - p)^T M (q - p), the key in exact arithmetic.
// Row k of the B operand holds (hi(psi), lo(psi), hi(psi), 0, 0), hi = psi
// with its low 13 mantissa bits cleared (a TF32 value), lo = psi - hi (exact);
// the search's A rows hold (hi(phi), hi(phi), lo(phi), 0, 0), so one K = 32
// TF32 product sums hi.hi + hi.lo + lo.hi.  Padding rows: psi = (0, .., 1e30).
// tcinfo: o (3) | 2^-12 max|psi_k| (10) | 1e-5 max nu (13) | max |p'|_1 (14)
// | 2^-20 max sum|M_ab| (15), nu = sum_a |sigma_a| |R_a|^2; entry 13 is +inf
// when a value of the tile is not finite (no bound: every point is a
// candidate).  The search turns these into its error bound.
__device__ void tc_tile_operand(const float* tile, float (*red)[8], int k, bool real, float* __restrict__ ops,
                                float* __restrict__ info) {
  __shared__ float red2[kTilePoints / 32][16];
  const int lane = k & 31, warp = k >> 5;
  float o[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float lo = INFINITY, hi = -INFINITY;
    for (int w = 0; w < kTilePoints / 32; ++w) {
      lo = fminf(lo, red[w][a]);
      hi = fmaxf(hi, red[w][3 + a]);
    }
    o[a] = (lo <= hi && isfinite(lo) && isfinite(hi)) ? 0.5f * lo + 0.5f * hi : 0.0f;
  }
  float psi[10];
  float nu = 0.f, lam = 0.f, p1 = 0.f;
  bool bad = false;
  if (real) {
    double r[kRecLen];
#pragma unroll
    for (int m = 0; m < kRecLen; ++m) r[m] = tile[m * kTilePoints + k];
    double pp[3], M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, nud = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) pp[a] = -r[kNPX + a] - (double)o[a];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double sg = r[kS0 + a];
      double rn = 0.0;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const double ra = r[kR00 + 3 * a + m];
        rn += ra * ra;
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) M[m][n2] += sg * ra * r[kR00 + 3 * a + n2];
      }
      nud += fabs(sg) * rn;
    }
    double mp[3], pmp = 0.0, lamd = 0.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      mp[m] = M[m][0] * pp[0] + M[m][1] * pp[1] + M[m][2] * pp[2];
      pmp += pp[m] * mp[m];
#pragma unroll
      for (int n2 = 0; n2 < 3; ++n2) lamd += fabs(M[m][n2]);
    }
    const double pd[10] = {M[0][0], M[1][1], M[2][2], 2 * M[0][1], 2 * M[0][2], 2 * M[1][2],
                           -2 * mp[0], -2 * mp[1], -2 * mp[2], pmp};
#pragma unroll
    for (int j = 0; j < 10; ++j) {
      psi[j] = (float)pd[j];
      if (!isfinite(psi[j])) bad = true;
    }
#pragma unroll
    for (int m = 0; m < kRecLen - 1; ++m)
      if (!isfinite(r[m])) bad = true;
    nu = (float)(nud * (1.0 + 1e-6));
    lam = (float)(lamd * (1.0 + 1e-6));
    p1 = (float)((fabs(pp[0]) + fabs(pp[1]) + fabs(pp[2])) * (1.0 + 1e-6));
    if (!isfinite(nu) || !isfinite(lam) || !isfinite(p1)) bad = true;
  } else {
#pragma unroll
    for (int j = 0; j < 9; ++j) psi[j] = 0.f;
    psi[9] = 1e30f;
  }
  // B row k: (hi, lo, hi, 0, 0) in the core-matrix layout: 8-row groups of
  // 8 chunks of 4 values, 128 B per (group, chunk)
  float row[kTcK];
#pragma unroll
  for (int j = 0; j < 10; ++j) {
    const float h = tf32_hi(psi[j]);
    row[j] = h;
    row[10 + j] = psi[j] - h;
    row[20 + j] = h;
  }
  row[30] = row[31] = 0.f;
  float4* dst = reinterpret_cast<float4*>(ops + (k >> 3) * (8 * 32) + (k & 7) * 4);
#pragma unroll
  for (int c = 0; c < kTcK / 4; ++c) dst[c * 8] = make_float4(row[4 * c], row[4 * c + 1], row[4 * c + 2], row[4 * c + 3]);
  // tile maxima of the bound terms over its real points
  float v[14];
#pragma unroll
  for (int j = 0; j < 10; ++j) v[j] = real ? fabsf(psi[j]) : 0.f;
  v[10] = nu;
  v[11] = p1;
  v[12] = lam;
  v[13] = bad ? 1.f : 0.f;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int j = 0; j < 14; ++j) v[j] = fmaxf(v[j], __shfl_xor_sync(0xffffffffu, v[j], off));
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < 14; ++j) red2[warp][j] = v[j];
  __syncthreads();
  if (k < kTcInfoFloats) {
    auto tmax = [&](int j) { return fmaxf(fmaxf(red2[0][j], red2[1][j]), fmaxf(red2[2][j], red2[3][j])); };
    const bool nonfinite = red2[0][13] != 0.f || red2[1][13] != 0.f || red2[2][13] != 0.f || red2[3][13] != 0.f;
    float out;
    if (k < 3) out = o[k];
    else if (k < 13) out = ldexpf(tmax(k - 3), -12);
    else if (k == 13) out = nonfinite ? INFINITY : 1e-5f * tmax(10);
    else if (k == 14) out = tmax(11);
    else out = ldexpf(tmax(12), -20);
    info[k] = out;
  }
}

// One CTA of 128 threads per search tile (tile blockIdx.x of group
// blockIdx.y), one sorted point per thread: packs the tile field-major --
// field f of point pair m (points 2m, 2m+1) at float2 f * 64 + m, so a lane
// reads its pair's 16 fields conflict-free and one packed f32x2 evaluation
// gives both keys -- (field kRecPad carries the original point index, -1
// for padding, whose sigma is NaN so its key is never a candidate) and
// writes tinfo[tile * kTinfoFloats]: the tile's {min xyz, max xyz, mu, 0},
// then one such box per warp's 32 points (the sub-boxes).
__global__ void __launch_bounds__(kTilePoints) tile_info_kernel(const float* __restrict__ rec,
                                                                const int* __restrict__ perm,
                                                                const CloudDesc* __restrict__ cd, int P, int ntile,
                                                                float* __restrict__ pairs,
                                                                float* __restrict__ tinfo,
                                                                float* __restrict__ tcops,
                                                                float* __restrict__ tcinfo) {
  const TileGroup g = tile_group(cd, blockIdx.y, P, ntile);
  const int t = blockIdx.x;
  if (t >= g.ntile) return;
  __shared__ float red[kTilePoints / 32][8];
  __shared__ __align__(16) float tile[kTilePoints * kRecLen];
  const int k = threadIdx.x, lane = k & 31, warp = k >> 5;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  float mu = INFINITY;
  bool bad = false;
  const int pos = t * kTilePoints + k;
  float* slot = tile + k;  // field f of point k at slot[f * kTilePoints]
  if (pos >= g.P) {
#pragma unroll
    for (int m = 0; m < kRecLen; ++m)
      slot[m * kTilePoints] = m == kRecPad ? __int_as_float(-1)
                                           : ((m == kS0 || m == kS1 || m == kS2) ? __int_as_float(0x7fc00000) : 0.0f);
  } else {
    const int idx = perm[g.p0 + pos];
    const float* r = rec + (g.p0 + idx) * kRecLen;
    float v[kRecLen];
    load_rec(r, v);
#pragma unroll
    for (int m = 0; m < kRecLen; ++m) slot[m * kTilePoints] = m == kRecPad ? __int_as_float(idx) : v[m];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float c = -v[kNPX + a];
      mn[a] = fminf(mn[a], c);
      mx[a] = fmaxf(mx[a], c);
      if (!isfinite(c)) bad = true;
    }
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double err = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double s = v[kS0 + a];
      if (!(s >= 0.0)) bad = true;  // a negative (or NaN) precision: keys may be negative
      double rn = 0.0;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const double ra = v[kR00 + 3 * a + m];
        rn += ra * ra;
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) M[m][n2] += s * ra * (double)v[kR00 + 3 * a + n2];
      }
      err += fabs(s) * rn;
    }
    const double lam = sym3_min_eig(M[0][0], M[1][1], M[2][2], M[0][1], M[0][2], M[1][2]);
    const double scale = fabs(M[0][0]) + fabs(M[1][1]) + fabs(M[2][2]) + fabs(M[0][1]) + fabs(M[0][2]) + fabs(M[1][2]);
    const double m = lam - 1e-9 * scale - 1e-5 * err;
    if (!isfinite(m)) bad = true;
    mu = fminf(mu, (m > 0.0 && isfinite(m)) ? (float)(m * (1.0 - 1e-6)) : 0.0f);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
      mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
    }
    mu = fminf(mu, __shfl_xor_sync(0xffffffffu, mu, o));
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    for (int a = 0; a < 3; ++a) {
      red[warp][a] = mn[a];
      red[warp][3 + a] = mx[a];
    }
    red[warp][6] = mu;
    red[warp][7] = bad ? 1.0f : 0.0f;
    float* o = tinfo + (g.t0 + t) * kTinfoFloats + 8 * (1 + warp);  // this warp's sub-box
    for (int a = 0; a < 3; ++a) {
      o[a] = mn[a];
      o[3 + a] = mx[a];
    }
    o[6] = bad ? -1.0f : mu;  // +inf: no points (the box is empty)
    o[7] = 0.0f;
  }
  __syncthreads();
  {
    const float4* src = reinterpret_cast<const float4*>(tile);
    float4* dst = reinterpret_cast<float4*>(pairs + (g.t0 + t) * kTilePoints * kRecLen);
    for (int i = k; i < kTilePoints * kRecLen / 4; i += kTilePoints) dst[i] = src[i];
  }
  if (tcops) tc_tile_operand(tile, red, k, pos < g.P, tcops + (g.t0 + t) * kTcOpsFloats, tcinfo + (g.t0 + t) * kTcInfoFloats);
  if (k == 0) {
    for (int w = 1; w < kTilePoints / 32; ++w) {
      for (int a = 0; a < 3; ++a) {
        mn[a] = fminf(mn[a], red[w][a]);
        mx[a] = fmaxf(mx[a], red[w][3 + a]);
      }
      mu = fminf(mu, red[w][6]);
      bad = bad || red[w][7] != 0.0f;
    }
    float* o = tinfo + (g.t0 + t) * kTinfoFloats;
    for (int a = 0; a < 3; ++a) {
      o[a] = mn[a];
      o[3 + a] = mx[a];
    }
    o[6] = bad ? -1.0f : (mu < INFINITY ? mu : 0.0f);  // -1: the tile has no key bound
    o[7] = 0.0f;
  }
}

int spatial_bits(int P) {
  int bits = 1;
  while (bits < 10 && (int64_t(1) << (3 * bits)) * 8 < P) ++bits;
  return bits;
}

namespace {
unsigned grid_x(int64_t n, int sms, int groups) {
  const int64_t cap = std::max<int64_t>(1, (int64_t)sms * 16 / std::max(1, groups));
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, cap));
}
}  // namespace

int launch_spatial_index(const float* q, const float* rec, int B, int Q, int P, int P_pad, char* ws, const FwdLayout& L,
                         cudaStream_t st, bool tc_ops) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int bits = L.bits, cells = 1 << (3 * bits);
  float* bnd = reinterpret_cast<float*>(ws + L.bounds);
  int* cnt = reinterpret_cast<int*>(ws + L.cell_count);
  int* off = reinterpret_cast<int*>(ws + L.cell_offset);
  int* perm = reinterpret_cast<int*>(ws + L.perm_p);  // perm_q follows perm_p directly
  float* pairs = reinterpret_cast<float*>(ws + L.pairs);
  float* tinfo = reinterpret_cast<float*>(ws + L.tinfo);
  const int ntile = P_pad / kTilePoints;
  GroupMap pm{P, bits, nullptr, nullptr, nullptr, nullptr, nullptr};
  GroupMap qm{Q, bits, nullptr, nullptr, nullptr, nullptr, nullptr};
  // the packing kernel wrote kBoundParts partial boxes per element (reduced
  // by the cell kernels) and zeroed the cell counts.  Points and queries in
  // one counting sort: their cells are scanned together, so the queries'
  // positions start after all points' and land in perm_q, which follows perm_p
  const int64_t nc = 2 * (int64_t)B * cells;
  const CellJob jp{rec + kNPX, kRecLen, 1, pm, 0, kBoundParts};
  const CellJob jq{q, 3, 0, qm, B * cells, kBoundParts, reinterpret_cast<int*>(ws + L.qseed), (int64_t)B * P};
  const dim3 grid(grid_x(P > Q ? P : Q, sms, B), B, 2);
  cell_count_kernel<<<grid, 256, 0, st>>>(jp, jq, bnd, cnt);
  if (nc <= kScatterScanMax) {
    // the packing kernel zeroed the offsets region too: it is the cursor here
    cell_scatter_scan_kernel<<<grid, 256, 0, st>>>(jp, jq, bnd, cnt, (int)nc, off, perm);
    note_launches(1);
  } else {
    int rc = launch_exclusive_scan(cnt, (int)nc, off, st);
    if (rc) return rc;
    cell_scatter_kernel<<<grid, 256, 0, st>>>(jp, jq, bnd, off, cnt, perm);
  }
  tile_info_kernel<<<dim3(ntile, B), kTilePoints, 0, st>>>(rec, perm, nullptr, P, ntile, pairs, tinfo,
                                                            tc_ops ? reinterpret_cast<float*>(ws + L.tcops) : nullptr,
                                                            tc_ops ? reinterpret_cast<float*>(ws + L.tcinfo) : nullptr);
  note_launches(3);  // + 1 scan, counted by launch_exclusive_scan
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

// Cloud-set index: bounds, Hilbert order, sorted tiles and tile boxes of
// every cloud (records already packed); the cell offsets stay in the cloud
// set.  Scratch: cell counts [total_cells], point permutation [total_p].
int launch_cloudset_index(char* cs, const CloudSetHeader& h, const CloudDesc* cd_dev, int max_p, int max_ntile,
                          int* cnt, int* perm_p, cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int C = h.C;
  const float* rec = reinterpret_cast<const float*>(cs + h.rec_off);
  int* off = reinterpret_cast<int*>(cs + h.celloff_off);
  float* bnd = reinterpret_cast<float*>(cs + h.bnd_off);
  float* pairs = reinterpret_cast<float*>(cs + h.pairs_off);
  float* tinfo = reinterpret_cast<float*>(cs + h.tinfo_off);
  GroupMap pm{0, 0, cd_dev, nullptr, nullptr, nullptr, nullptr};
  point_bounds_kernel<<<C, 512, 0, st>>>(rec, pm, bnd);
  if (cudaMemsetAsync(cnt, 0, (size_t)h.total_cells * 4, st) != cudaSuccess) return KNNAG_ERR_CUDA;
  const CellJob jp{rec + kNPX, kRecLen, 1, pm, 0, 0};
  const dim3 grid(grid_x(max_p, sms, C), C, 1);
  cell_count_kernel<<<grid, 256, 0, st>>>(jp, jp, bnd, cnt);
  int rc = launch_exclusive_scan(cnt, h.total_cells, off, st);
  if (rc) return rc;
  cell_scatter_kernel<<<grid, 256, 0, st>>>(jp, jp, bnd, off, cnt, perm_p);
  tile_info_kernel<<<dim3(max_ntile, C), kTilePoints, 0, st>>>(rec, perm_p, cd_dev, 0, 0, pairs, tinfo, nullptr,
                                                                nullptr);
  note_launches(4);  // + 1 scan
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

// Query order of a segment table: every segment's queries counting-sorted by
// the Hilbert index of a grid cell over its cloud's box.  cnt/off hold cap_cells
// (+1) cells (the encoded total is at most that); perm_q gets, at each
// segment's rows, the segment-local query indices in sorted order.  Sizes
// come from the device copy of the table, so the launches replay on new
// tables of the same capacity.
int launch_query_order(const float* q, const char* cs, const void* segs_dev, int cap_segs, int64_t cap_q,
                       int cap_cells, int* cnt, int* off, int* perm_q, const int* status, cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  GroupMap qm{0, 0, nullptr, seg_descs(segs_dev), static_cast<const SegHeader*>(segs_dev), cs, status};
  if (cudaMemsetAsync(cnt, 0, (size_t)cap_cells * 4, st) != cudaSuccess) return KNNAG_ERR_CUDA;
  const dim3 grid(grid_x(cap_q, sms, cap_segs), cap_segs, 1);
  const CellJob jq{q, 3, 0, qm, 0, 0};
  cell_count_kernel<<<grid, 256, 0, st>>>(jq, jq, nullptr, cnt);
  int rc = launch_exclusive_scan(cnt, cap_cells, off, st);
  if (rc) return rc;
  cell_scatter_kernel<<<grid, 256, 0, st>>>(jq, jq, nullptr, off, cnt, perm_q);
  note_launches(2);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

}  // namespace knnag
