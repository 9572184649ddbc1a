// lowprec.cuh -- device helpers for the FP32 / FP16 storage formats of
// mixed.cuh: link and colour-vector loads and stores, two-row (12-real)
// long-link reconstruction and the sign a long link carries.
#pragma once
#include <cuda_fp16.h>

#include "internal.cuh"
#include "mixed.cuh"

namespace qs {

constexpr int kF32 = 0;
constexpr int kF16 = 1;  // 16-bit fixed point (see h2f)

// 16-bit storage is fixed point: a 16-bit integer per real, scaled by a
// per-site norm (colour vectors) or a per-list scale (links) so that the
// largest magnitude maps to 32767.  This keeps 15 bits of resolution
// relative to the largest element, where an IEEE half keeps 11.  The integer
// i in [-32767, 32767] is stored in offset binary, u = i + 32768, so that a
// load needs no int->float conversion instruction (those run on the
// quarter-rate XU pipe and bounded the Dslash): one byte permute places u in
// the low mantissa bits of 2^23 and one FP32 add subtracts 2^23 + 32768,
// exactly, on full-rate pipes.
constexpr float kI16 = 32767.f;
// raw integers of a packed pair, as floats (no scaling)
__device__ __forceinline__ float2 h2f(unsigned w) {
  const float lo = __uint_as_float(__byte_perm(w, 0x4B00u, 0x5410)) - 8421376.0f;
  const float hi = __uint_as_float(__byte_perm(w, 0x4B00u, 0x5432)) - 8421376.0f;
  return make_float2(lo, hi);
}
// pack two values in [-1, 1]
__device__ __forceinline__ unsigned f2h(float a, float b) {
  int ia = __float2int_rn(fminf(fmaxf(a, -1.f), 1.f) * kI16) + 32768;
  int ib = __float2int_rn(fminf(fmaxf(b, -1.f), 1.f) * kI16) + 32768;
  return ((unsigned)ia & 0xffffu) | ((unsigned)ib << 16);
}

// Link pointers of one handle as the kernels see them.
struct LoLinks {
  const float4 *f32_fat;
  const float2 *f32_fat_tail;
  const float4 *f32_long;
  const float2 *f32_long_tail;
  const uint4 *f16_fat;
  const unsigned *f16_fat_tail;
  const uint4 *f16_long;
  const uint2 *f16_long_tail2;
  const unsigned *f16_long_tail;
  float fat_scale;   // value of one raw 16-bit unit of fat (or naive) links; 1 for FP32
  float long_scale;  // value of one raw 16-bit unit of long links; 1 for FP32
  float long_rc;     // row-2 factor of a 12-real long link: long_scale / long_coeff
  int recon12;
};

// Staggered phase sign of a long link of direction mu at x (forward) and at
// x - 3 mu (backward): eta_mu(x) (QEX phases [8,9,11,0]; eta_mu does not
// depend on x_mu) times -1 where the three-hop link crosses the
// antiperiodic time boundary.  On a domain's slab the boundary is the
// global one: slice x3 is global slice (x3 + t0) mod L3g (t0 is even, so
// eta is the same in either coordinate).
__device__ __forceinline__ float eta_sign(int mu, const int x[4]) {
  int s = (mu == 0) ? x[3] : (mu == 1) ? (x[0] + x[3]) : (mu == 2) ? (x[0] + x[1] + x[3]) : 0;
  return (s & 1) ? -1.f : 1.f;
}
__device__ __forceinline__ int global_t(const Geom &g, int x3) {
  int t = x3 + g.t0;
  if (t >= g.L3g) t -= g.L3g;
  if (t < 0) t += g.L3g;
  return t;
}
__device__ __forceinline__ float long_sign_fwd(const Geom &g, const int x[4], int mu) {
  float s = eta_sign(mu, x);
  return (mu == 3 && global_t(g, x[3]) + 3 >= g.L3g) ? -s : s;
}
__device__ __forceinline__ float long_sign_bck(const Geom &g, const int x[4], int mu) {
  float s = eta_sign(mu, x);
  return (mu == 3 && global_t(g, x[3]) < 3) ? -s : s;
}

// row 2 = k * conj(row0 x row1)
__device__ __forceinline__ void recon_row2(float2 u[9], float k) {
  const float2 a0 = u[0], a1 = u[1], a2 = u[2], b0 = u[3], b1 = u[4], b2 = u[5];
  // (a x b)_i = a_j b_k - a_k b_j
  float2 c0 = make_float2(a1.x * b2.x - a1.y * b2.y - (a2.x * b1.x - a2.y * b1.y),
                          a1.x * b2.y + a1.y * b2.x - (a2.x * b1.y + a2.y * b1.x));
  float2 c1 = make_float2(a2.x * b0.x - a2.y * b0.y - (a0.x * b2.x - a0.y * b2.y),
                          a2.x * b0.y + a2.y * b0.x - (a0.x * b2.y + a0.y * b2.x));
  float2 c2 = make_float2(a0.x * b1.x - a0.y * b1.y - (a1.x * b0.x - a1.y * b0.y),
                          a0.x * b1.y + a0.y * b1.x - (a1.x * b0.y + a1.y * b0.x));
  u[6] = make_float2(k * c0.x, -k * c0.y);
  u[7] = make_float2(k * c1.x, -k * c1.y);
  u[8] = make_float2(k * c2.x, -k * c2.y);
}

// 18-real link f of a list at site
template <int PREC>
__device__ __forceinline__ void load_link18(const float4 *c32, const float2 *t32, const uint4 *c16,
                                            const unsigned *t16, int f, size_t site, size_t V,
                                            float2 u[9]) {
  if (PREC == kF32) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float4 q = ldlink(c32 + ((size_t)f * 4 + j) * V + site);
      u[2 * j] = make_float2(q.x, q.y);
      u[2 * j + 1] = make_float2(q.z, q.w);
    }
    u[8] = ldlink(t32 + (size_t)f * V + site);
  } else {
#pragma unroll
    for (int j = 0; j < 2; j++) {
      uint4 q = ldlink(c16 + ((size_t)f * 2 + j) * V + site);
      u[4 * j] = h2f(q.x);
      u[4 * j + 1] = h2f(q.y);
      u[4 * j + 2] = h2f(q.z);
      u[4 * j + 3] = h2f(q.w);
    }
    u[8] = h2f(ldlink(t16 + (size_t)f * V + site));
  }
}

// 12-real long link f at site, row 2 rebuilt with sign s
template <int PREC>
__device__ __forceinline__ void load_long12(const LoLinks &L, int f, size_t site, size_t V, float s,
                                            float2 u[9]) {
  if (PREC == kF32) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float4 q = ldlink(L.f32_long + ((size_t)f * 3 + j) * V + site);
      u[2 * j] = make_float2(q.x, q.y);
      u[2 * j + 1] = make_float2(q.z, q.w);
    }
  } else {
    uint4 q = ldlink(L.f16_long + (size_t)f * V + site);
    uint2 t = ldlink(L.f16_long_tail2 + (size_t)f * V + site);
    u[0] = h2f(q.x);
    u[1] = h2f(q.y);
    u[2] = h2f(q.z);
    u[3] = h2f(q.w);
    u[4] = h2f(t.x);
    u[5] = h2f(t.y);
  }
  recon_row2(u, s * L.long_rc);
}

// colour vectors: FP32 float2[3][stride]; 16-bit uint4[stride]
template <int PREC>
__device__ __forceinline__ void load_vec(const void *base, int stride, int i, float2 v[3]) {
  if (PREC == kF32) {
    const float2 *p = (const float2 *)base;
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = ldg(p + (size_t)c * stride + i);
  } else {
    uint4 q = ldg((const uint4 *)base + i);
    float n = __uint_as_float(q.w) * (1.f / kI16);
    float2 a = h2f(q.x), b = h2f(q.y), c = h2f(q.z);
    v[0] = make_float2(n * a.x, n * a.y);
    v[1] = make_float2(n * b.x, n * b.y);
    v[2] = make_float2(n * c.x, n * c.y);
  }
}
// same, coherent (the vector may be written by the same kernel elsewhere)
template <int PREC>
__device__ __forceinline__ void load_vec_cg(const void *base, int stride, int i, float2 v[3]) {
  if (PREC == kF32) {
    const float2 *p = (const float2 *)base;
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = __ldcg(p + (size_t)c * stride + i);
  } else {
    uint4 q = __ldcg((const uint4 *)base + i);
    float n = __uint_as_float(q.w) * (1.f / kI16);
    float2 a = h2f(q.x), b = h2f(q.y), c = h2f(q.z);
    v[0] = make_float2(n * a.x, n * a.y);
    v[1] = make_float2(n * b.x, n * b.y);
    v[2] = make_float2(n * c.x, n * c.y);
  }
}

template <int PREC>
__device__ __forceinline__ void store_vec(void *base, int stride, int i, const float2 v[3]) {
  if (PREC == kF32) {
    float2 *p = (float2 *)base;
#pragma unroll
    for (int c = 0; c < 3; c++) p[(size_t)c * stride + i] = v[c];
  } else {
    float n = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) n = fmaxf(n, fmaxf(fabsf(v[c].x), fabsf(v[c].y)));
    const float inv = n > 0.f ? 1.f / n : 0.f;
    uint4 q;
    q.x = f2h(v[0].x * inv, v[0].y * inv);
    q.y = f2h(v[1].x * inv, v[1].y * inv);
    q.z = f2h(v[2].x * inv, v[2].y * inv);
    q.w = __float_as_uint(n);
    ((uint4 *)base)[i] = q;
  }
}

// ---- packed-pair forms for the 16-bit Dslash (sm_100 FP32x2 instructions) ----
//
// The colour sums there are built as t_i = T_i + i S_i with
// T_i = sum_j u_ij * Re v_j and S_i = sum_j u_ij * Im v_j, each term one
// FP32x2 FMA of the link element's (re, im) pair with a vector component
// broadcast to both lanes.

// raw integers of a packed 16-bit pair as (sx re, sy im): exact, one FP32x2
// op after the two byte permutes (sx, sy = +-1 fold a negation or a
// conjugation into the decode)
template <int SX, int SY>
__device__ __forceinline__ float2 h2f2(unsigned w) {
  constexpr float B = 8421376.0f;  // 2^23 + 32768
  const float2 r = make_float2(__uint_as_float(__byte_perm(w, 0x4B00u, 0x5410)),
                               __uint_as_float(__byte_perm(w, 0x4B00u, 0x5432)));
  if (SX == 1 && SY == 1) return __fadd2_rn(r, make_float2(-B, -B));
  return __ffma2_rn(r, make_float2((float)SX, (float)SY), make_float2(-SX * B, -SY * B));
}

// 18-real 16-bit link f at site as (re, im) pairs, times (SX, SY) per pair
template <int SX, int SY>
__device__ __forceinline__ void load_link18_x2(const uint4 *c16, const unsigned *t16, int f, size_t site,
                                               size_t V, float2 u[9]) {
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const uint4 q = ldlink(c16 + ((size_t)f * 2 + j) * V + site);
    u[4 * j] = h2f2<SX, SY>(q.x);
    u[4 * j + 1] = h2f2<SX, SY>(q.y);
    u[4 * j + 2] = h2f2<SX, SY>(q.z);
    u[4 * j + 3] = h2f2<SX, SY>(q.w);
  }
  u[8] = h2f2<SX, SY>(ldlink(t16 + (size_t)f * V + site));
}

// 12-real 16-bit long link f at site, times (SX, SY), row 2 rebuilt with k
template <int SX, int SY>
__device__ __forceinline__ void load_long12_x2(const LoLinks &L, int f, size_t site, size_t V, float k,
                                               float2 u[9]) {
  const uint4 q = ldlink(L.f16_long + (size_t)f * V + site);
  const uint2 t = ldlink(L.f16_long_tail2 + (size_t)f * V + site);
  u[0] = h2f2<SX, SY>(q.x);
  u[1] = h2f2<SX, SY>(q.y);
  u[2] = h2f2<SX, SY>(q.z);
  u[3] = h2f2<SX, SY>(q.w);
  u[4] = h2f2<SX, SY>(t.x);
  u[5] = h2f2<SX, SY>(t.y);
  recon_row2(u, k);
}

// colour vector at i as broadcast pairs br[c] = s Re v_c (both lanes),
// bi[c] = s Im v_c
template <int VP>
__device__ __forceinline__ void load_vec_bc(const void *base, int stride, int i, float s, float2 br[3],
                                            float2 bi[3]) {
  if (VP == kF32) {
    const float2 *p = (const float2 *)base;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 v = ldg(p + (size_t)c * stride + i);
      br[c] = make_float2(s * v.x, s * v.x);
      bi[c] = make_float2(s * v.y, s * v.y);
    }
  } else {
    const uint4 q = ldg((const uint4 *)base + i);
    const float n = __uint_as_float(q.w) * (1.f / kI16) * s;
    const unsigned w[3] = {q.x, q.y, q.z};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 r = h2f2<1, 1>(w[c]);
      br[c] = __fmul2_rn(make_float2(r.x, r.x), make_float2(n, n));
      bi[c] = __fmul2_rn(make_float2(r.y, r.y), make_float2(n, n));
    }
  }
}

// bytes of one site of a colour vector in each format
constexpr int vec_bytes(int prec) { return prec == kF32 ? 24 : 16; }

LoLinks lo_links(const LowLinks &low, int prec);

}  // namespace qs
