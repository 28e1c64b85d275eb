// Tensor-core filtered kNN search + aggregation: uniform FP32 calls, K <= 32.
//
// Replaces the search half of csrc/forward.cu:83-95 and the aggregation of
// csrc/forward.cu:100-109 (one thread per query scanning every point) with
//
//   1. approximate keys of 128 queries x 128 points per search tile from one
//      tcgen05.mma (kind::tf32, M = N = 128, K = 32) into TMEM.  With the
//      tile's origin o, the key (q - p)^T M (q - p), M = R^T diag(sigma) R, is
//      phi(q - o) . psi(p - o) for 10 quadratic / linear / constant features
//      (knn_spatial.cu, tc_tile_operand); each feature is split into a TF32
//      high part and an FP32 remainder, and the K = 32 product sums
//      hi.hi + hi.lo + lo.hi, accurate to about 2^-20 of sum |phi_k psi_k|;
//   2. a rigorous bound E(q, tile) on |approximate - exact| (the GEMM's error
//      with a 32x margin, the rounding of the exact FP32 key, the rounding of
//      q - o); a point is a candidate when its approximate key is at most
//      the query's threshold + E (NaN: always), so every point whose exact
//      key is at most the threshold is a candidate;
//   3. the exact FP32 key (the reference's contraction, bit for bit) of each
//      candidate from the tile's records in shared memory, inserted into the
//      query's sorted register list of K+1 (the threshold is the list top, or
//      the query's seed while that is smaller).
//
// Results are the CUDA-core search's: the same list, the same exactness
// flags (ties, empty slots, NaN in MinK's fill phase -> the exact replay),
// the same epilogue.  One CTA of 256 threads holds 128 sorted queries (one
// TMEM lane and two threads each); tiles arrive by 1-D bulk copies (no multicast) on
// mbarriers with bounded waits; the TMEM accumulator (128 columns) is
// allocated at the start and freed on every exit path.
#include <math.h>

#include "knn_common.cuh"
#include "knn_internal.h"
#include "knn_search_dev.cuh"

namespace knnag {
namespace {

constexpr int kTcQ = 128;           // queries per CTA = MMA M = TMEM lanes
constexpr int kTcThreads = 256;     // two threads per query
constexpr uint32_t kTcCols = 128;   // TMEM columns: one 128 x 128 FP32 accumulator
// tcgen05.mma kind::tf32 instruction descriptor: D F32 (bits 4-5 = 1), A and
// B TF32 (bits 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

// Shared memory of a CTA.
constexpr size_t kTcOffB = 0;                                      // B operand ring, 2 x 16 KB
constexpr size_t kTcOffR = kTcOffB + 2 * (size_t)kTcOpsBytes;      // record tiles, 2 x 8 KB
constexpr size_t kTcOffA = kTcOffR + 2 * kSearchTileBytes;         // A operand, 16 KB
constexpr size_t kTcOffTI = kTcOffA + kTcOpsBytes;                 // tile boxes, 2 x 160 B
constexpr size_t kTcOffTC = kTcOffTI + 2 * (size_t)kTinfoBytes;    // bound terms, 2 x 64 B
constexpr size_t kTcOffQT = kTcOffTC + 2 * (size_t)kTcInfoBytes;   // [128] float4 (x, y, z, seed)
constexpr size_t kTcOffQO = kTcOffQT + (size_t)kTcQ * 16;          // [128] original query index
constexpr size_t kTcOffTop = kTcOffQO + (size_t)kTcQ * 4;          // [2][256] list tops
constexpr size_t kTcOffMisc = kTcOffTop + 2 * (size_t)kTcThreads * 4;  // barriers, TMEM address, flags
constexpr size_t kTcFixed = kTcOffMisc + 256;                      // then tile bounds + visit order
// At most 4 CTAs fit an SM by shared memory, so 4 x 128 TMEM columns never
// exceed the SM's 512: an allocation never waits for another CTA.
static_assert(kTcFixed * 5 > (size_t)228 * 1024, "TMEM columns could be oversubscribed");
static_assert((size_t)kTcQ * 33 * 12 + kTcQ * 4 <= kTcOffTI, "epilogue staging exceeds the operand region");
static_assert((size_t)kTcThreads * 4 * 2 >= (size_t)kTcQ * 4, "tie keys of the second lists exceed the tops region");

__host__ __device__ inline size_t tc_smem_bytes(int ntile) { return kTcFixed + search_region_c_bytes(ntile); }

// ------------------------------------------------------------ tcgen05 PTX
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[adesc] x B[bdesc]^T, issued by one thread.
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}
// Arrive on `bar` once every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Shared-memory matrix descriptor of a K-major operand without swizzle:
// core matrices of 8 rows x 16 B stored contiguously (128 B); the two core
// matrices of one K = 8 step are 128 B apart (leading byte offset), 8-row
// groups 1024 B apart (stride byte offset); version 1 (bit 46).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         (1ull << 46);
}

// 32 consecutive columns of this thread's TMEM lane, waited for in the same
// statement (so no use of the values can be scheduled before the wait).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 64 consecutive columns of this thread's TMEM lane (one load, then the wait).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, "
      "%37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, "
      "%59, %60, %61, %62, %63}, [%64];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]),
        "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]),
        "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]),
        "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]),
        "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 64; ++j) v[j] = __uint_as_float(r[j]);
}

// Exact key of point pt of a record tile in shared memory (field f of point
// pt at rt[f * kTilePoints + pt]) and the point's original index.
__device__ __forceinline__ float tile_key(float qx, float qy, float qz, const float* rt, int pt, int& idx) {
  const float* r = rt + pt;
  float rr[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) rr[i] = r[(kR00 + i) * kTilePoints];
  const float x = add_rn(qx, r[kNPX * kTilePoints]);
  const float y = add_rn(qy, r[kNPY * kTilePoints]);
  const float z = add_rn(qz, r[kNPZ * kTilePoints]);
  idx = __float_as_int(r[kRecPad * kTilePoints]);
  return key_from_offset(x, y, z, rr, r[kS0 * kTilePoints], r[kS1 * kTilePoints], r[kS2 * kTilePoints]);
}

// ------------------------------------------------------------------ kernel
// Thread t of the CTA's 256 serves sorted query qs = t % 128 (TMEM lane qs:
// warps w and w + 4 share TMEM sub-partition w) and half h = t / 128 of
// every tile (points 64h .. 64h + 63).  Each of a query's two threads keeps
// its own sorted list; both use the smaller list top (and the seed) as the
// threshold -- either top bounds the union's (K+1)-th smallest key from
// above -- and the lists are merged at the end.
template <int KMAX>
__global__ void __launch_bounds__(kTcThreads, KMAX <= 16 ? 2 : 1) search_tc_kernel(SearchParams a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr int L = KMAX + 1;
  constexpr int NT = kTcQ;
  constexpr int NTH = kTcThreads;
  constexpr unsigned FULL = 0xffffffffu;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int qs = tid & (kTcQ - 1), half = tid / kTcQ, sub = warp & 3;

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTcOffMisc);  // [0], [1] tile copies; [2] MMA done
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + kTcOffMisc + 32);
  volatile int* s_ncand = reinterpret_cast<volatile int*>(smem + kTcOffMisc + 36);
  volatile int* s_fillok = reinterpret_cast<volatile int*>(smem + kTcOffMisc + 40);
  float* qbox = reinterpret_cast<float*>(smem + kTcOffMisc + 48);    // [4][6]
  float* s_wmax = reinterpret_cast<float*>(smem + kTcOffMisc + 144);  // [2][8]
  float4* qtab = reinterpret_cast<float4*>(smem + kTcOffQT);
  int* qorig = reinterpret_cast<int*>(smem + kTcOffQO);
  float* s_top = reinterpret_cast<float*>(smem + kTcOffTop);         // [2][256] list tops
  const int ntp_cap = search_tiles_pow2(a.ntile);
  float* lbk = reinterpret_cast<float*>(smem + kTcFixed);
  int* lbt = reinterpret_cast<int*>(lbk + ntp_cap);

  // TMEM accumulator (warp 0) and the barriers (thread 0)
  if (warp == 0) {
    tmem_alloc(s_tmem, kTcCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  // the plan's item (batch element, sorted query range) when the plan ran,
  // else block (blockIdx.x, blockIdx.y) of 128 queries
  int64_t b = blockIdx.y;
  int q0 = blockIdx.x * kTcQ, q1 = min(q0 + kTcQ, a.Q);
  if (a.items) {
    const int4 itm = a.items[blockIdx.x];
    b = itm.x;
    q0 = itm.y;
    q1 = itm.z;
  }
  const int Q = a.Q, P = a.P, K = a.K, ntile = a.ntile;
  const float* rec_b = a.rec + b * P * kRecLen;
  const float* pairs_b = a.pairs + b * (a.P_pad / 2) * kPairFloats;
  const float* tinfo_b = a.tinfo + b * ntile * kTinfoFloats;
  const float* tcops_b = a.tcops + b * ntile * kTcOpsFloats;
  const float* tcinfo_b = a.tcinfo + b * ntile * kTcInfoFloats;

  // ---- this thread's query (sorted position sp of batch element b)
  const int sp = q0 + qs;
  bool valid = sp < q1;
  int qi = a.perm_q[b * Q + (valid ? sp : Q - 1)];
  if ((unsigned)qi >= (unsigned)Q) {  // the query order is a permutation: never taken
    if (valid && half == 0) atomicOr(a.status, kStatusBadIndex);
    qi = 0;
    valid = false;
  }
  const float* qrow = a.q + (b * Q + qi) * 3;
  const float qx = qrow[0], qy = qrow[1], qz = qrow[2];
  const float qpt[3] = {qx, qy, qz};
  if (half == 0) {
    qorig[qs] = valid ? qi : -1;
    qtab[qs] = make_float4(qx, qy, qz, valid ? INFINITY : -INFINITY);
  }
  // MinK's fill phase keeps points 0..K-1 whatever their key, so a NaN key
  // there needs the replay.  With those records finite and below 1e6 in
  // magnitude, and the query too, no key can overflow or be NaN; otherwise
  // the keys are evaluated.
  if (warp == 0) {
    bool ok = true;
    if (lane < K) {
      float r[kRecLen];
      load_rec(rec_b + (int64_t)lane * kRecLen, r);
#pragma unroll
      for (int m = 0; m < kRecLen - 1; ++m) ok = ok && fabsf(r[m]) <= 1e6f;  // NaN fails
    }
    ok = __all_sync(FULL, ok);
    if (lane == 0) *s_fillok = ok ? 1 : 0;
  }
  __syncthreads();
  if (a.items) {
    // seeds from the plan kernel
    if (half == 0 && valid) qtab[qs].w = a.tau0[b * Q + sp];
  } else {
    // seeds: warp w computes those of queries 32 (w % 4) + 16 h .. + 15
    const int g0 = 32 * sub + 16 * half;
    const int sq = g0 + (lane & 15);
    const int ssp = q0 + sq;
    const bool sval = lane < 16 && qorig[sq] >= 0;
    const int my_seed = sval ? a.qseed[b * Q + ssp] : 0;
    seed_warp<KMAX, 16>(qtab + g0, my_seed, sval, pairs_b, P, K, lane);
  }
  bool nan_fill = false;
  if (half == 0 && valid && !(*s_fillok && fabsf(qx) <= 1e6f && fabsf(qy) <= 1e6f && fabsf(qz) <= 1e6f))
    for (int i = 0; i < K; ++i) {
      const float s = key_rec<float>(qx, qy, qz, rec_b + (int64_t)i * kRecLen);
      if (s != s) nan_fill = true;
    }
  if (tid == 0) *s_ncand = 0;
  __syncthreads();

  // ---- the CTA's query box, the tiles below its largest seed, ascending
  if (half == 0) {
    float bx[6] = {qx, qy, qz, qx, qy, qz};
    if (!valid) {
      bx[0] = bx[1] = bx[2] = INFINITY;
      bx[3] = bx[4] = bx[5] = -INFINITY;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bx[c] = fminf(bx[c], __shfl_xor_sync(FULL, bx[c], o));
        bx[3 + c] = fmaxf(bx[3 + c], __shfl_xor_sync(FULL, bx[3 + c], o));
      }
    float tw = valid ? qtab[qs].w : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tw = fmaxf(tw, __shfl_xor_sync(FULL, tw, o));
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) qbox[warp * 6 + c] = bx[c];
      s_wmax[warp] = tw;
    }
  }
  __syncthreads();
  float bmin[3], bmax[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    bmin[c] = fminf(fminf(qbox[c], qbox[6 + c]), fminf(qbox[12 + c], qbox[18 + c]));
    bmax[c] = fmaxf(fmaxf(qbox[3 + c], qbox[9 + c]), fmaxf(qbox[15 + c], qbox[21 + c]));
  }
  float tmax = fmaxf(fmaxf(s_wmax[0], s_wmax[1]), fmaxf(s_wmax[2], s_wmax[3]));
  for (int t = tid; t < ntile; t += NTH) {
    const float lb = tile_lower_bound(tinfo_b + (int64_t)t * kTinfoFloats, bmin, bmax);
    if (!(lb > tmax)) {
      const int pos = atomicAdd(const_cast<int*>(s_ncand), 1);
      lbk[pos] = fminf(lb, 3.4e38f);
      lbt[pos] = t;
    }
  }
  __syncthreads();
  const int nv = *s_ncand;
  if (nv <= 32) {
    // (bound, tile) ascending in warp 0's registers (shuffle bitonic network)
    if (warp == 0) {
      float lb = lane < nv ? lbk[lane] : INFINITY;
      int ti = lane < nv ? lbt[lane] : 0x7fffffff;
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
      if (lane < nv) {
        lbk[lane] = lb;
        lbt[lane] = ti;
      }
    }
  } else {
    // bitonic sort in shared memory over the next power of two
    const int ns = search_tiles_pow2(nv);  // <= ntp_cap
    for (int t = nv + tid; t < ns; t += NTH) {
      lbk[t] = INFINITY;
      lbt[t] = 0x7fffffff;
    }
    __syncthreads();
    for (int kk = 2; kk <= ns; kk <<= 1) {
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
  __syncthreads();

  // ---- tile loop
  float keys[L];
  int vals[L];
#pragma unroll
  for (int s = 0; s < L; ++s) {
    keys[s] = (s < KMAX - K) ? -INFINITY : INFINITY;
    vals[s] = -1;
  }
  const float seed = valid ? qtab[qs].w : -INFINITY;
  float tau = seed, tie_key = INFINITY;

  unsigned char* ring_b = smem + kTcOffB;
  unsigned char* ring_r = smem + kTcOffR;
  float* amat = reinterpret_cast<float*>(smem + kTcOffA);
  const uint32_t a_saddr = smem_u32(amat);
  auto issue = [&](int v) {
    const int slot = v & 1;
    const int64_t t = lbt[v];
    mbar_arrive_expect_tx(&bars[slot], kTcOpsBytes + (uint32_t)kSearchTileBytes + kTinfoBytes + kTcInfoBytes);
    if (v == a.stall_visit) return;  // test hook: this phase never completes
    bulk_copy_g2s(ring_b + slot * kTcOpsBytes, tcops_b + t * kTcOpsFloats, kTcOpsBytes, &bars[slot]);
    bulk_copy_g2s(ring_r + slot * kSearchTileBytes, pairs_b + t * (kTilePoints / 2) * kPairFloats,
                  (uint32_t)kSearchTileBytes, &bars[slot]);
    bulk_copy_g2s(smem + kTcOffTI + slot * kTinfoBytes, tinfo_b + t * kTinfoFloats, kTinfoBytes, &bars[slot]);
    bulk_copy_g2s(smem + kTcOffTC + slot * kTcInfoBytes, tcinfo_b + t * kTcInfoFloats, kTcInfoBytes, &bars[slot]);
  };
  // One CTA barrier per tile.  Visit v: wait for its copy, write the A rows,
  // publish the list tops; barrier; then thresholds are refreshed, visit
  // v + 1 is issued into the other slot (every thread is past visit v - 1),
  // and the MMA and the readout of visit v run.  The MMA of visit v + 1 is
  // issued only after the next barrier, which every thread reaches after its
  // readout of visit v, so one TMEM accumulator and one A buffer suffice.
  // s_abort[v & 1] collects the failed waits that the barrier of visit v
  // must see: the copy of visit v and the MMA of visit v - 1 (flags only
  // ever go from 0 to 1)
  volatile int* s_abort = reinterpret_cast<volatile int*>(smem + kTcOffMisc + 208);
  int issued = 0;  // visits issued (thread 0's count)
  if (tid == 0) {
    s_abort[0] = s_abort[1] = 0;
    fence_proxy_async_smem();  // this CTA's generic shared-memory accesses before the copies
    if (nv > 0) {
      if ((unsigned)lbt[0] >= (unsigned)ntile) {  // real tiles sort first: never taken
        atomicOr(a.status, kStatusBadIndex);
      } else {
        issue(0);
        issued = 1;
      }
    }
  }
  __syncthreads();
  int limit = nv < 1 ? nv : 1;  // visits known (to every thread) to have been issued
  bool aborted = false;
  int nmma = 0, v = 0;
  for (; v < limit; ++v) {
    if (lbk[v] > tmax) break;  // every later tile is above every threshold
    const int slot = v & 1;
    const bool ok_copy = mbar_wait_bounded(&bars[slot], (v >> 1) & 1, a.wait_spins);
    if (!ok_copy) {
      if (lane == 0) atomicOr(a.status, kStatusWaitTimeout);
      s_abort[v & 1] = 1;
    }
    const float* ti = reinterpret_cast<const float*>(smem + kTcOffTI + slot * kTinfoBytes);
    const float* tc = reinterpret_cast<const float*>(smem + kTcOffTC + slot * kTcInfoBytes);
    const bool need_t = ok_copy && valid && !(tile_lower_bound(ti, qpt, qpt) > tau);
    // this thread's half of the query's A row: phi(q - o) as (hi, hi, lo,
    // 0, 0), chunks 4h .. 4h + 3; and the error bound
    float E;
    {
      const float x = __fsub_rn(qx, tc[0]), y = __fsub_rn(qy, tc[1]), z = __fsub_rn(qz, tc[2]);
      float ph[10] = {x * x, y * y, z * z, x * y, x * z, y * z, x, y, z, 1.f};
      if (!valid) {
#pragma unroll
        for (int j = 0; j < 10; ++j) ph[j] = 0.f;
      }
      const float q1 = fabsf(x) + fabsf(y) + fabsf(z);
      float e1 = 0.f;
#pragma unroll
      for (int j = 0; j < 10; ++j) e1 = fmaf(fabsf(ph[j]), tc[3 + j], e1);
      const float s1 = q1 + tc[14];
      E = (e1 + tc[13] * s1 * s1 + tc[15] * q1 * s1 + 1e-30f) * 1.001f;
      float row[kTcK];
#pragma unroll
      for (int j = 0; j < 10; ++j) {
        const float h = tf32_hi(ph[j]);
        row[j] = h;
        row[10 + j] = h;
        row[20 + j] = ph[j] - h;
      }
      row[30] = row[31] = 0.f;
      float4* dst = reinterpret_cast<float4*>(amat + (qs >> 3) * (8 * 32) + (qs & 7) * 4);
      if (half == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[c * 8] = make_float4(row[4 * c], row[4 * c + 1], row[4 * c + 2], row[4 * c + 3]);
      } else {
#pragma unroll
        for (int c = 4; c < 8; ++c) dst[c * 8] = make_float4(row[4 * c], row[4 * c + 1], row[4 * c + 2], row[4 * c + 3]);
      }
    }
    // the list top after the previous visit, for the partner thread and the
    // CTA's largest threshold
    const float mytop = keys[L - 1];
    s_top[(v & 1) * NTH + tid] = mytop;
    {
      float tw = valid ? fminf(tau, mytop) : -INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tw = fmaxf(tw, __shfl_xor_sync(FULL, tw, o));
      if (lane == 0) s_wmax[(v & 1) * 8 + warp] = tw;
    }
    fence_proxy_async_smem();  // the A rows are read by the tensor core (async proxy)
    const int any = __syncthreads_or(need_t);
    if (s_abort[v & 1]) {
      aborted = true;
      if (ok_copy) ++v;  // this visit's copy was waited for (by every thread whose wait succeeded)
      break;
    }
    tau = fminf(fminf(tau, mytop), s_top[(v & 1) * NTH + (tid ^ kTcQ)]);
    {
      const float* wm = s_wmax + (v & 1) * 8;
      float tm = -INFINITY;
#pragma unroll
      for (int w = 0; w < 8; ++w) tm = fmaxf(tm, wm[w]);
      tmax = fminf(tmax, tm);  // a query's threshold is the smaller of its two threads'
    }
    if (v + 1 < nv && !(lbk[v + 1] > tmax)) {
      if (tid == 0) {
        if ((unsigned)lbt[v + 1] >= (unsigned)ntile) {
          atomicOr(a.status, kStatusBadIndex);
        } else {
          fence_proxy_async_smem();
          issue(v + 1);
          issued = v + 2;
        }
      }
      limit = v + 2;
    }
    if (any) {
      if (tid == 0) {
        tc_fence_after();
        const uint32_t b_saddr = smem_u32(ring_b + slot * kTcOpsBytes);
#pragma unroll
        for (int k = 0; k < kTcK / 8; ++k) tc_mma(tmem, tc_desc(a_saddr + 256 * k), tc_desc(b_saddr + 256 * k), k > 0);
        tc_commit(&bars[2]);
      }
      const bool ok_mma = mbar_wait_bounded(&bars[2], nmma & 1, a.wait_spins);
      ++nmma;
      if (!ok_mma) {
        if (lane == 0) atomicOr(a.status, kStatusWaitTimeout);
        s_abort[(v + 1) & 1] = 1;  // acted on at the next barrier
      }
      tc_fence_after();
      const float* rt = reinterpret_cast<const float*>(ring_r + slot * kSearchTileBytes);
      const bool need_h = need_t && ok_mma &&
                          !(fminf(tile_lower_bound(ti + 8 * (1 + 2 * half), qpt, qpt),
                                  tile_lower_bound(ti + 8 * (2 + 2 * half), qpt, qpt)) > tau);
      if (__any_sync(FULL, need_h)) {
        float av[64];
        tmem_ld64(tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(half * 64), av);
        if (need_h) {
          const float bnd = tau + E;
          uint32_t m0 = 0, m1 = 0;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            m0 |= (av[j] > bnd ? 0u : 1u) << j;
            m1 |= (av[32 + j] > bnd ? 0u : 1u) << j;
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            uint32_t m = u ? m1 : m0;
            while (m) {
              const int j = __ffs(m) - 1;
              m &= m - 1;
              int idx;
              const float sk = tile_key(qx, qy, qz, rt, half * 64 + u * 32 + j, idx);
              const float top = keys[L - 1];
              if (sk < top) {
                list_insert<L>(keys, vals, sk, idx, tie_key);
              } else if (sk == top) {
                tie_key = fminf(tie_key, sk);
              }
            }
          }
          tau = fminf(tau, keys[L - 1]);
        }
      }
      tc_fence_before();
    }
  }
  if (!aborted) {
    // a failed MMA wait of the last visit: no barrier followed it yet
    __syncthreads();
    if (s_abort[0] || s_abort[1]) aborted = true;
  }
  // Every copy issued lands before the CTA leaves or reuses the ring (the
  // loop may stop with one or two visits in flight); a wait that gives up
  // has latched the timeout already.
  __syncthreads();
  if (tid == 0) {
    for (int u = v; u < issued; ++u) mbar_wait_bounded(&bars[u & 1], (u >> 1) & 1, a.wait_spins);
    if (aborted && nmma > 0) mbar_wait_bounded(&bars[2], (nmma - 1) & 1, a.wait_spins);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTcCols);
  }
  if (aborted) return;

  // ---- merge each query's second list into its first (the same insertion
  // and tie rules as the candidates), then flags and staging; the operand
  // region is free now
  float* out_k = reinterpret_cast<float*>(smem);
  int* out_i = reinterpret_cast<int*>(out_k + NT * L);
  float* out_w = reinterpret_cast<float*>(out_i + NT * L);
  int* out_f = reinterpret_cast<int*>(out_w + NT * L);
  float* tie_s = reinterpret_cast<float*>(smem + kTcOffTop);  // the second lists' tie keys
  if (half == 1) {
#pragma unroll
    for (int s = 0; s < L; ++s) {
      out_k[qs * L + s] = keys[s];
      out_i[qs * L + s] = vals[s];
    }
    tie_s[qs] = tie_key;
  }
  __syncthreads();
  if (half == 0) {
    tie_key = fminf(tie_key, tie_s[qs]);
    for (int s = KMAX - K; s < L; ++s) {
      const int i = out_i[qs * L + s];
      if (i < 0) continue;  // empty slot
      const float k = out_k[qs * L + s];
      const float top = keys[L - 1];
      if (k < top) {
        list_insert<L>(keys, vals, k, i, tie_key);
      } else if (k == top) {
        tie_key = fminf(tie_key, k);
      }
    }
  }
  __syncthreads();
  if (half == 0) {
#pragma unroll
    for (int s = 0; s < L; ++s) {
      const int j = s - (KMAX - K);
      if (j >= 0) {
        out_k[qs * L + j] = keys[s];
        out_i[qs * L + j] = vals[s];
      }
    }
    const int nneed = (P > K) ? K + 1 : K;
    bool fl = nan_fill, bad = false;
    for (int j = 0; j < nneed; ++j) {
      const int idx = out_i[qs * L + j];
      if (idx < 0) fl = true;
      if (idx >= P) bad = true;  // tiles carry indices of their own cloud: never taken
    }
    if (bad && valid) atomicOr(a.status, kStatusBadIndex);
    for (int j = 0; j + 1 < nneed; ++j)
      if (out_k[qs * L + j] == out_k[qs * L + j + 1]) fl = true;
    const float m = (P > K) ? out_k[qs * L + K] : INFINITY;
    if (tie_key <= m) fl = true;
    for (int j = 0; j < K; ++j) out_w[qs * L + j] = weight_of(out_k[qs * L + j]);
    out_f[qs] = (fl || bad || !valid) ? 1 : 0;
    if (valid && fl && !bad) {
      const int pos = atomicAdd(a.flag_count, 1);
      a.flag_list[pos] = (int)(b * Q + qi);
    }
  }
  __syncthreads();

  // ---- epilogue: dists / idxs / w_out, then f_out = sum_k w_k f[idx_k] in
  // k order with fma, 128-bit gathers of f rows, to the queries' rows
  float* dists = a.dists + b * Q * K;
  int64_t* idxs = a.idxs + b * Q * K;
  float* w_out = a.w_out + b * Q * K;
  int* adj = a.adj_count ? a.adj_count + b * P : nullptr;
  for (int x = tid; x < NT * K; x += NTH) {
    const int l = x / K, k = x - l * K;
    if (out_f[l]) continue;
    const int64_t e = (int64_t)qorig[l] * K + k;
    const int idx = out_i[l * L + k];
    dists[e] = out_k[l * L + k];
    idxs[e] = (int64_t)idx;
    w_out[e] = out_w[l * L + k];
    if (adj) atomicAdd(&adj[idx], 1);  // idx is in [0, P): unflagged
  }
  const int F = a.F;
  const float* fb = a.f + b * P * F;
  float* fo = a.f_out + b * Q * F;
  if (a.vec4) {
    const int C4 = F >> 2;
    for (int x = tid; x < NT * C4; x += NTH) {
      const int l = x / C4, c = x - l * C4;
      if (out_f[l]) continue;
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      constexpr int RB = 16;  // rows in flight, summed in k order
      for (int k0 = 0; k0 < K; k0 += RB) {
        float4 vv[RB];
        float w[RB];
#pragma unroll
        for (int j = 0; j < RB; ++j) {
          const bool in = k0 + j < K;
          const int idx = in ? out_i[l * L + k0 + j] : 0;
          w[j] = in ? out_w[l * L + k0 + j] : 0.f;
          vv[j] = in ? __ldg(reinterpret_cast<const float4*>(fb + (int64_t)idx * F) + c) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < RB; ++j) {
          if (k0 + j < K) {
            acc.x = __fmaf_rn(vv[j].x, w[j], acc.x);
            acc.y = __fmaf_rn(vv[j].y, w[j], acc.y);
            acc.z = __fmaf_rn(vv[j].z, w[j], acc.z);
            acc.w = __fmaf_rn(vv[j].w, w[j], acc.w);
          }
        }
      }
      reinterpret_cast<float4*>(fo + (int64_t)qorig[l] * F)[c] = acc;
    }
  } else {
    for (int x = tid; x < NT * F; x += NTH) {
      const int l = x / F, c = x - l * F;
      if (out_f[l]) continue;
      float acc = 0.f;
      for (int k = 0; k < K; ++k) acc = __fmaf_rn(__ldg(fb + (int64_t)out_i[l * L + k] * F + c), out_w[l * L + k], acc);
      fo[(int64_t)qorig[l] * F + c] = acc;
    }
  }
}

template <int KMAX>
int launch_tc_t(const SearchParams& a0, cudaStream_t st) {
  const size_t smem = tc_smem_bytes(a0.ntile);
  if (smem > 227 * 1024) return KNNAG_ERR_TOO_LARGE;
  static int attr_set[64] = {0};  // largest size already allowed, per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && attr_set[dev] < (int)smem) {
    if (cudaFuncSetAttribute(search_tc_kernel<KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return KNNAG_ERR_CUDA;
    attr_set[dev] = (int)smem;
  }
  // Grids of more than one wave run the search plan first (seeds and the
  // blocks' tile estimates, then the blocks ordered heaviest first), so the
  // last waves hold light blocks; in one wave every block starts at once.
  const int nb = (a0.Q + kTcQ - 1) / kTcQ;
  const int64_t nbt = (int64_t)nb * a0.B;
  SearchParams a = a0;
  const bool plan = a.items && a.tau0 && a.plan_est && nbt <= search_plan_max_blocks() &&
                    nbt > (int64_t)(KMAX <= 16 ? 2 : 1) * num_sms(dev);
  if (!plan) a.items = nullptr;
  const dim3 grid = plan ? dim3((unsigned)nbt, 1) : dim3((unsigned)nb, (unsigned)a.B);
  profile_begin(st);  // the plan does the seed work of the search: timed with it
  if (plan) {
    const int rc = launch_search_plan(a, kTcQ, nb, st);
    if (rc) {
      profile_end(st);
      return rc;
    }
  }
  search_tc_kernel<KMAX><<<grid, kTcThreads, smem, st>>>(a);
  profile_end(st);
  note_launches(1);
  return cudaGetLastError() == cudaSuccess ? KNNAG_OK : KNNAG_ERR_CUDA;
}

}  // namespace

bool search_tc_fits(int ntile) { return tc_smem_bytes(ntile) <= 227 * 1024; }

int launch_search_tc(const SearchParams& a, cudaStream_t st) {
  if (!a.tcops || !a.tcinfo || a.K < 1 || a.K > 32 || a.B > 65535) return KNNAG_ERR_ARG;
  if (tc_smem_bytes(a.ntile) > 227 * 1024) return KNNAG_ERR_TOO_LARGE;
  if (a.K <= 8) return launch_tc_t<8>(a, st);
  if (a.K <= 16) return launch_tc_t<16>(a, st);
  return launch_tc_t<32>(a, st);
}

}  // namespace knnag
