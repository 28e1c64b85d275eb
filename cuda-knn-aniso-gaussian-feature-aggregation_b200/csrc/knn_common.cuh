// Shared device/host definitions for the anisotropic kNN aggregation kernels.
//
// Key arithmetic.  For a query q and point i the reference computes
// (csrc/forward.cu:85-92)
//     x = q0 - p0, y = q1 - p1, z = q2 - p2
//     j = R00*x + R01*y + R02*z   (k, l likewise with rows 1 and 2)
//     s = j*j*s0 + k*k*s1 + l*l*s2
// and nvcc (-fmad=true) contracts it to
//     j = fma(R02, z, fma(R00, x, R01*y))
//     s = fma(l*l, s2, fma(j*j, s0, (k*k)*s1))
// -- pinned bit for bit against the reference extension on a B200 over 2.7M
// keys.  Every key below is written with explicit round-to-nearest
// intrinsics in exactly that order so the compiler cannot re-contract it;
// x is formed as q + (-p) from pre-negated coordinates, which IEEE defines
// to be the same value as q - p.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "knn_aniso.h"

namespace knnag {

// ---------------------------------------------------------------- records
// Per-point record (16 values of T): the packed form every kernel gathers.
enum RecField {
  kNPX = 0, kNPY = 1, kNPZ = 2,   // -p
  kR00 = 3,                       // R row-major, 9 values: kR00 + 3*row + col
  kS0 = 12, kS1 = 13, kS2 = 14,   // sigma
  kRecPad = 15,
  kRecLen = 16
};

// Points per search tile (8 KB) and the floats of one point pair (2m, 2m+1)
// in it: 16 fields x float2.  Tiles are field-major (field f of pair m at
// float2 f * 64 + m), so packed f32x2 arithmetic reads both points' field
// with one load and a warp reads 32 pairs' field with one conflict-free load.
constexpr int kTilePoints = 128;
// Per search tile: {min xyz, max xyz, mu, 0} of the tile's box, then the same
// for each of its 32-point sub-boxes (sorted points 32w .. 32w + 31); mu is
// the key lower-bound factor of the points inside (-1: no bound, +inf with
// the empty box: no points).
constexpr int kSubBoxes = kTilePoints / 32;
constexpr int kTinfoFloats = 8 * (1 + kSubBoxes);
constexpr unsigned kTinfoBytes = kTinfoFloats * 4;
constexpr int kPairFloats = 32;
// Tensor-core filter, per search tile: the B operand of the approximate-key
// GEMM (128 points x 32 TF32 values in the no-swizzle K-major core-matrix
// layout, 16 KB) and 16 floats of error-bound terms (origin, feature
// bounds, rounding factors).
constexpr int kTcK = 32;
constexpr int kTcOpsFloats = kTilePoints * kTcK;
constexpr unsigned kTcOpsBytes = kTcOpsFloats * 4;
constexpr int kTcInfoFloats = 16;
constexpr unsigned kTcInfoBytes = kTcInfoFloats * 4;

__host__ __device__ inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------- status
// Word 0 of every workspace: device-side error latch.  Word 1: number of
// queries flagged for the exact MinK replay.
constexpr int kStatusWaitTimeout = 1;
constexpr int kStatusBadTable = 2;  // a segment table entry the kernel cannot serve
constexpr int kStatusBadIndex = 4;  // an internal index out of range (self-check; the access was skipped)

// ---------------------------------------------------------------- keys
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// One rotated coordinate u = r0*x + r1*y + r2*z in the reference's rounding.
template <typename T>
__device__ __forceinline__ T row_dot(T r0, T r1, T r2, T x, T y, T z) {
  return fma_rn(r2, z, fma_rn(r0, x, mul_rn(r1, y)));
}

// s = j*j*s0 + k*k*s1 + l*l*s2 in the reference's rounding.
template <typename T>
__device__ __forceinline__ T quad_form(T j, T k, T l, T s0, T s1, T s2) {
  return fma_rn(mul_rn(l, l), s2, fma_rn(mul_rn(j, j), s0, mul_rn(mul_rn(k, k), s1)));
}

// Key from an already formed offset (x, y, z) and a row-major R.
template <typename T>
__device__ __forceinline__ T key_from_offset(T x, T y, T z, const T* r, T s0, T s1, T s2) {
  const T j = row_dot(r[0], r[1], r[2], x, y, z);
  const T k = row_dot(r[3], r[4], r[5], x, y, z);
  const T l = row_dot(r[6], r[7], r[8], x, y, z);
  return quad_form(j, k, l, s0, s1, s2);
}

// A point record (16 values, 64 B in FP32 / 128 B in FP64, 16-byte
// aligned) into registers with 128-bit loads: four (eight) load
// instructions per record instead of fifteen scalar ones.
__device__ __forceinline__ void load_rec(const float* p, float (&r)[kRecLen]) {
  const float4* v = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int i = 0; i < kRecLen / 4; ++i) {
    const float4 x = __ldg(v + i);
    r[4 * i + 0] = x.x;
    r[4 * i + 1] = x.y;
    r[4 * i + 2] = x.z;
    r[4 * i + 3] = x.w;
  }
}
__device__ __forceinline__ void load_rec(const double* p, double (&r)[kRecLen]) {
  const double2* v = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int i = 0; i < kRecLen / 2; ++i) {
    const double2 x = __ldg(v + i);
    r[2 * i + 0] = x.x;
    r[2 * i + 1] = x.y;
  }
}

// Key of query (qx,qy,qz) against a per-point record in global memory.
template <typename T>
__device__ __forceinline__ T key_rec(T qx, T qy, T qz, const T* rec_g) {
  T rec[kRecLen];
  load_rec(rec_g, rec);
  T x = add_rn(qx, rec[kNPX]);
  T y = add_rn(qy, rec[kNPY]);
  T z = add_rn(qz, rec[kNPZ]);
  return key_from_offset(x, y, z, rec + kR00, rec[kS0], rec[kS1], rec[kS2]);
}

// Packed key of one query (duplicated into both halves of qx2..) against a
// point pair: 18 packed FP32 instructions for two keys.
__device__ __forceinline__ float2 key_pair(float2 qx2, float2 qy2, float2 qz2, const float2* pr) {
  float2 x = __fadd2_rn(qx2, pr[kNPX]);
  float2 y = __fadd2_rn(qy2, pr[kNPY]);
  float2 z = __fadd2_rn(qz2, pr[kNPZ]);
  const float2* r = pr + kR00;
  float2 j = __ffma2_rn(r[2], z, __ffma2_rn(r[0], x, __fmul2_rn(r[1], y)));
  float2 k = __ffma2_rn(r[5], z, __ffma2_rn(r[3], x, __fmul2_rn(r[4], y)));
  float2 l = __ffma2_rn(r[8], z, __ffma2_rn(r[6], x, __fmul2_rn(r[7], y)));
  return __ffma2_rn(__fmul2_rn(l, l), pr[kS2],
                    __ffma2_rn(__fmul2_rn(j, j), pr[kS0], __fmul2_rn(__fmul2_rn(k, k), pr[kS1])));
}

// The TF32 part of x (low 13 mantissa bits cleared); x - tf32_hi(x) is exact.
__device__ __forceinline__ float tf32_hi(float x) { return __int_as_float(__float_as_int(x) & 0xffffe000); }

// Weight of a key: the reference's fast-math __expf in FP32
// (csrc/forward.cu:102); full-precision exp in FP64.
__device__ __forceinline__ float weight_of(float s) { return __expf(-s); }
__device__ __forceinline__ double weight_of(double s) { return exp(-s); }

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait suspends the thread in hardware until the phase completes or a
// short time limit passes.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Plain arrival (count 1, no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Default spin budget of mbar_wait_bounded: about a second of 256 ns sleeps.
constexpr int kWaitSpinsDefault = 1 << 22;

// Wait for phase `parity` of `bar` to complete, giving up after `spins`
// sleeps of 256 ns (after 256 hardware-suspended tries); returns false on
// timeout (the caller latches the error and leaves).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int spins = kWaitSpinsDefault) {
  for (int spin = 0; spin < 256; ++spin)
    if (mbar_try_wait(bar, parity)) return true;
  for (int spin = 0; spin < spins; ++spin) {
    if (mbar_test_wait(bar, parity)) return true;
    __nanosleep(256);
  }
  return false;
}

// 1-D bulk copy global -> shared completing on `bar` (bytes % 16 == 0,
// both addresses 16-byte aligned).  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------ Hilbert grid cells

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Position of grid cell (x, y, z) (bits bits per axis) along the 3-D Hilbert
// curve, by J. Skilling's transpose algorithm ("Programming the Hilbert
// curve", AIP Conf. Proc. 707, 2004): undo the excess work, Gray-encode,
// then interleave the transposed coordinates (X[0] most significant).
// Consecutive cells along the curve are always face neighbours, so a run of
// sorted points (a search tile) or queries (a CTA) stays compact; the
// Z-order curve jumps across the box at every level.
__device__ __forceinline__ uint32_t hilbert3(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  return (spread3(X[0]) << 2) | (spread3(X[1]) << 1) | spread3(X[2]);
}

__device__ __forceinline__ uint32_t cell_of(float x, float y, float z, const float* bnd, int bits) {
  const float res = (float)(1 << bits);
  uint32_t c[3];
  const float v[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = bnd[a], ext = bnd[3 + a] - bnd[a];
    float t = ext > 0.f ? (v[a] - lo) / ext * res : 0.f;
    t = fminf(fmaxf(t, 0.f), res - 1.f);  // NaN -> 0
    c[a] = (uint32_t)t;
  }
  return hilbert3(c[0], c[1], c[2], bits);
}

}  // namespace knnag
