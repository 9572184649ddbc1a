// mixed.cuh -- reduced-precision storage formats used by the sloppy inner
// solvers.  All arrays are structure-of-arrays over the site index so that a
// warp's loads of one chunk are contiguous 16-byte words.
//
//  FP32 link, 18 reals:   float4 [n][4][V] (elements 0..7) + float2 [n][V] (element 8)
//  FP32 long link, 12 reals (rows 0 and 1): float4 [n][3][V]
//  16-bit link, 18 reals: uint4 [n][2][V] (elements 0..7, one re/im pair of
//                          int16 per 32-bit word) + unsigned [n][V] (element 8);
//                          value = int16 / 32767 * scale, scale = max |real| of the list
//  16-bit long link, 12 reals: uint4 [n][V] (elements 0..3) + uint2 [n][V] (4..5)
//  FP32 vector:           float2 [3][stride]
//  16-bit vector:         uint4 [stride] = (c0, c1, c2 as int16 re/im pairs, float norm),
//                          value = int16 / 32767 * norm, norm = max |real| of the site
// The 16-bit formats are what the API calls half precision (SLOPPY_HALF):
// 16-bit fixed point with FP32 scales, computed in FP32.
//
// A 12-real long link stores rows 0 and 1 of W = s*c*U, U in SU(3), s = +-1 the
// folded phase/boundary sign of that link and c the long-link coefficient.
// Row 2 is rebuilt as (s/c) * conj(row0 x row1); s is recomputed from the
// site coordinates (QEX phases [8,9,11,0] and the antiperiodic time
// boundary), so no sign needs storing.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace qs {

struct LowLinks {
  bool ready = false;
  bool recon12 = false;   // long links stored with 12 reals
  int nfat = 0, nlong = 0;  // naive: nfat = 4, nlong = 0
  double long_coeff = 1.0;
  // FP32
  float4 *f32_fat = nullptr;
  float2 *f32_fat_tail = nullptr;
  float4 *f32_long = nullptr;       // recon12: [nlong][3][V]; else [nlong][4][V]
  float2 *f32_long_tail = nullptr;  // only without recon12
  // FP16
  uint4 *f16_fat = nullptr;
  unsigned *f16_fat_tail = nullptr;
  uint4 *f16_long = nullptr;         // recon12: [nlong][V]; else [nlong][2][V]
  uint2 *f16_long_tail2 = nullptr;   // recon12 tail
  unsigned *f16_long_tail = nullptr; // without recon12
  float fat_scale = 1.0f, long_scale = 1.0f;
};

}  // namespace qs
