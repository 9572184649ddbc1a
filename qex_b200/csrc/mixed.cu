// mixed.cu -- reduced-precision link copies, the FP32 / FP16 Dslash and the
// reliable-update mixed-precision CG.
//
// Mixed-precision CG.  QEX's own sloppy solve (stagSolve.nim:101-117) is an
// FP32 CG inside FP64 defect correction, floored at FP32 epsilon.  Here the
// inner solver is a reliable-update CG (Sleijpen and van der Vorst 1996, the
// scheme QUDA uses): iterate in the sloppy precision, keep the solution
// increment in FP32, and whenever the iterated residual has dropped by delta
// since the last update (or the solve appears converged) fold the increment
// into the FP64 solution, recompute the true FP64 residual b - A x with the
// FP64 operator, restart the sloppy residual from it and re-orthogonalise
// the search direction.  All dot products and norms accumulate in FP64.
// The FP64 defect-correction loop of solveXX wraps this solver unchanged.
//
// Sloppy Dslash traffic per output site, fat+Naik with 12-real long links:
//   FP32: 4*(72+72)+4*(48+48) links + 24 in + 24 out = 1008 B
//   FP16: 4*(36+36)+4*(24+24) links + 16 in + 16 out = 512 B
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "lib.cuh"
#include "lowprec.cuh"

namespace qs {

// ---------------------------------------------------------------------------
// building the reduced-precision copies
// ---------------------------------------------------------------------------

__global__ void absmax_kernel(const double2 *__restrict__ u, size_t n, unsigned *out) {
  float m = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double2 v = u[i];
    m = fmaxf(m, (float)fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // m >= 0: uint order = float order
}

// max over long links of |row2 - (s/c) conj(row0 x row1)| / |c|
__global__ void recon_check_kernel(Geom g, const double2 *__restrict__ u64, double c, unsigned *out) {
  const size_t V = g.V;
  float m = 0.f;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 4 * g.V; t += gridDim.x * blockDim.x) {
    const int mu = t / g.V, site = t - mu * g.V;
    const int par = site >= g.nh ? 1 : 0;
    int x[4], lex;
    site_coords(g, par, site - par * g.nh, x, lex);
    double s = long_sign_fwd(g, x, mu);
    const double2 *ul = u64 + (size_t)(2 * mu + 1) * 9 * V + site;
    double2 e[9];
    for (int j = 0; j < 9; j++) e[j] = ul[(size_t)j * V];
    double2 cr[3];
    for (int i = 0; i < 3; i++) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      double2 a = e[j], b = e[3 + k], a2 = e[k], b2 = e[3 + j];
      cr[i] = make_double2(a.x * b.x - a.y * b.y - (a2.x * b2.x - a2.y * b2.y),
                           a.x * b.y + a.y * b.x - (a2.x * b2.y + a2.y * b2.x));
    }
    double k = s / c, d = 0;
    for (int i = 0; i < 3; i++) {
      d = fmax(d, fabs(e[6 + i].x - k * cr[i].x));
      d = fmax(d, fabs(e[6 + i].y + k * cr[i].y));
    }
    m = fmaxf(m, (float)(d / fabs(c)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// FP32/FP16 copy of link k (all sites) into list slot f
__global__ void to_low18_kernel(const double2 *__restrict__ uk, size_t V, float4 *c32, float2 *t32,
                                uint4 *c16, unsigned *t16, int f, float inv16) {
  for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < V; s += (size_t)gridDim.x * blockDim.x) {
    double2 e[9];
    for (int j = 0; j < 9; j++) e[j] = uk[(size_t)j * V + s];
    for (int j = 0; j < 4; j++)
      c32[((size_t)f * 4 + j) * V + s] =
          make_float4((float)e[2 * j].x, (float)e[2 * j].y, (float)e[2 * j + 1].x, (float)e[2 * j + 1].y);
    t32[(size_t)f * V + s] = make_float2((float)e[8].x, (float)e[8].y);
    for (int j = 0; j < 2; j++) {
      uint4 q;
      q.x = f2h((float)(e[4 * j].x * inv16), (float)(e[4 * j].y * inv16));
      q.y = f2h((float)(e[4 * j + 1].x * inv16), (float)(e[4 * j + 1].y * inv16));
      q.z = f2h((float)(e[4 * j + 2].x * inv16), (float)(e[4 * j + 2].y * inv16));
      q.w = f2h((float)(e[4 * j + 3].x * inv16), (float)(e[4 * j + 3].y * inv16));
      c16[((size_t)f * 2 + j) * V + s] = q;
    }
    t16[(size_t)f * V + s] = f2h((float)(e[8].x * inv16), (float)(e[8].y * inv16));
  }
}

__global__ void to_low12_kernel(const double2 *__restrict__ uk, size_t V, float4 *c32, uint4 *c16,
                                uint2 *t16, int f, float inv16) {
  for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < V; s += (size_t)gridDim.x * blockDim.x) {
    double2 e[6];
    for (int j = 0; j < 6; j++) e[j] = uk[(size_t)j * V + s];
    for (int j = 0; j < 3; j++)
      c32[((size_t)f * 3 + j) * V + s] =
          make_float4((float)e[2 * j].x, (float)e[2 * j].y, (float)e[2 * j + 1].x, (float)e[2 * j + 1].y);
    uint4 q;
    q.x = f2h((float)(e[0].x * inv16), (float)(e[0].y * inv16));
    q.y = f2h((float)(e[1].x * inv16), (float)(e[1].y * inv16));
    q.z = f2h((float)(e[2].x * inv16), (float)(e[2].y * inv16));
    q.w = f2h((float)(e[3].x * inv16), (float)(e[3].y * inv16));
    c16[(size_t)f * V + s] = q;
    uint2 t;
    t.x = f2h((float)(e[4].x * inv16), (float)(e[4].y * inv16));
    t.y = f2h((float)(e[5].x * inv16), (float)(e[5].y * inv16));
    t16[(size_t)f * V + s] = t;
  }
}

template <class T>
static int dalloc(T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "device allocation of reduced-precision links failed");
  }
  return QEXSTAG_OK;
}

static int read_uint(unsigned *d, unsigned *h) {
  QS_CUDA(cudaMemcpyAsync(h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

static int absmax_links(const double2 *u, size_t n, float *out, unsigned *scratch) {
  QS_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned), stream()));
  absmax_kernel<<<grid_for((long)std::min<size_t>(n, 1u << 30)), kBlock, 0, stream()>>>(u, n, scratch);
  note_launch();
  QS_LAUNCH_CHECK();
  unsigned h = 0;
  int rc = read_uint(scratch, &h);
  if (rc) return rc;
  float f;
  std::memcpy(&f, &h, sizeof(f));
  *out = f;
  return QEXSTAG_OK;
}

int build_low_links(qexstag_links_s *g) {
  LowLinks &L = g->low;
  L = LowLinks();
  const Geom &geo = g->l->g;
  const size_t V = geo.V;
  const bool naik = g->nl == 8;
  L.nfat = 4;
  L.nlong = naik ? 4 : 0;
  L.long_coeff = g->long_coeff;
  unsigned *scratch = (unsigned *)red_tickets() + (kNumTickets - 1);
  int rc;
  // scales (max |element|) of the fat and long lists
  float fat_max = 0.f, long_max = 0.f;
  for (int k = 0; k < g->nl; k++) {
    float m = 0.f;
    if ((rc = absmax_links(g->u64 + (size_t)k * 9 * V, 9 * V, &m, scratch))) return rc;
    if (naik && (k & 1))
      long_max = std::max(long_max, m);
    else
      fat_max = std::max(fat_max, m);
  }
  if (!(fat_max > 0.f) || !std::isfinite(fat_max) || (naik && (!(long_max > 0.f) || !std::isfinite(long_max))))
    return fail(QEXSTAG_ERR_ARG, "links_create: links are zero or not finite");
  L.fat_scale = fat_max;
  L.long_scale = naik ? long_max : 1.0f;
  // are the long links coeff * sign * SU(3)?
  if (naik) {
    QS_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned), stream()));
    recon_check_kernel<<<grid_for(4L * V), kBlock, 0, stream()>>>(geo, g->u64, g->long_coeff, scratch);
    note_launch();
    QS_LAUNCH_CHECK();
    unsigned h = 0;
    if ((rc = read_uint(scratch, &h))) return rc;
    float dev;
    std::memcpy(&dev, &h, sizeof(dev));
    L.recon12 = dev < 2e-6f;
  }
  if ((rc = dalloc(&L.f32_fat, (size_t)4 * 4 * V)) || (rc = dalloc(&L.f32_fat_tail, (size_t)4 * V)) ||
      (rc = dalloc(&L.f16_fat, (size_t)4 * 2 * V)) || (rc = dalloc(&L.f16_fat_tail, (size_t)4 * V)))
    return rc;
  for (int f = 0; f < 4; f++) {
    const int k = naik ? 2 * f : f;
    to_low18_kernel<<<grid_for((long)V), kBlock, 0, stream()>>>(g->u64 + (size_t)k * 9 * V, V, L.f32_fat,
                                                                L.f32_fat_tail, L.f16_fat, L.f16_fat_tail,
                                                                f, 1.0f / L.fat_scale);
    note_launch();
  }
  if (naik) {
    if (L.recon12) {
      if ((rc = dalloc(&L.f32_long, (size_t)4 * 3 * V)) || (rc = dalloc(&L.f16_long, (size_t)4 * V)) ||
          (rc = dalloc(&L.f16_long_tail2, (size_t)4 * V)))
        return rc;
      for (int f = 0; f < 4; f++) {
        to_low12_kernel<<<grid_for((long)V), kBlock, 0, stream()>>>(g->u64 + (size_t)(2 * f + 1) * 9 * V, V,
                                                                    L.f32_long, L.f16_long, L.f16_long_tail2,
                                                                    f, 1.0f / L.long_scale);
        note_launch();
      }
    } else {
      if ((rc = dalloc(&L.f32_long, (size_t)4 * 4 * V)) || (rc = dalloc(&L.f32_long_tail, (size_t)4 * V)) ||
          (rc = dalloc(&L.f16_long, (size_t)4 * 2 * V)) || (rc = dalloc(&L.f16_long_tail, (size_t)4 * V)))
        return rc;
      for (int f = 0; f < 4; f++) {
        to_low18_kernel<<<grid_for((long)V), kBlock, 0, stream()>>>(g->u64 + (size_t)(2 * f + 1) * 9 * V, V,
                                                                    L.f32_long, L.f32_long_tail, L.f16_long,
                                                                    L.f16_long_tail, f, 1.0f / L.long_scale);
        note_launch();
      }
    }
  }
  QS_LAUNCH_CHECK();
  L.ready = true;
  return QEXSTAG_OK;
}

void free_low_links(LowLinks &low) {
  cudaFree(low.f32_fat);
  cudaFree(low.f32_fat_tail);
  cudaFree(low.f32_long);
  cudaFree(low.f32_long_tail);
  cudaFree(low.f16_fat);
  cudaFree(low.f16_fat_tail);
  cudaFree(low.f16_long);
  cudaFree(low.f16_long_tail2);
  cudaFree(low.f16_long_tail);
  low = LowLinks();
}

LoLinks lo_links(const LowLinks &low, int prec) {
  LoLinks L;
  L.f32_fat = low.f32_fat;
  L.f32_fat_tail = low.f32_fat_tail;
  L.f32_long = low.f32_long;
  L.f32_long_tail = low.f32_long_tail;
  L.f16_fat = low.f16_fat;
  L.f16_fat_tail = low.f16_fat_tail;
  L.f16_long = low.f16_long;
  L.f16_long_tail2 = low.f16_long_tail2;
  L.f16_long_tail = low.f16_long_tail;
  L.recon12 = low.recon12 ? 1 : 0;
  if (prec == kF16) {
    L.fat_scale = low.fat_scale / kI16;
    L.long_scale = low.long_scale / kI16;
    L.long_rc = (float)((double)low.long_scale / kI16 / low.long_coeff);
  } else {
    L.fat_scale = 1.f;
    L.long_scale = 1.f;
    L.long_rc = (float)(1.0 / low.long_coeff);
  }
  return L;
}

// ---------------------------------------------------------------------------
// mixed-precision CG state
// ---------------------------------------------------------------------------

struct MxState {
  double r2;     // iterated (sloppy) |r|^2, or the true one after an update
  double r2old;  // |r|^2 of the previous iteration
  double alpha, beta, pAp, rp;
  double b2, r2req, r2stop, delta;
  double rNorm, r0Norm, maxrx, maxrr;
  int itn, maxits, done, pending, nan, reliable;
  int pin;     // p buffer (0 or 1) the last fused update read: the direction a reliable update corrects
  int itc[2];  // iterations done, as the fused update of host parity c reads (itc[c]) and writes (itc[c ^ 1])
  int pad;
};

__device__ __forceinline__ bool mx_halt(const MxState *st) { return st->done || st->pending; }

// Layout of the reduction scratch (red_partials) in the mixed CG: per-block
// <p, Ap> partials from 0, the update's |r|^2 partials from kMxR2, the half
// sweep's |Ap|^2 partials from kMxApAp, the fused update's second set of
// |r|^2 partials from kMxR2b (it reads one set and writes the other), the
// 16-bit half sweep's Re <r, Ap> partials from kMxRAp
constexpr int kMxR2 = kMaxRedBlocks, kMxApAp = 2 * kMaxRedBlocks, kMxR2b = 3 * kMaxRedBlocks,
              kMxRAp = 4 * kMaxRedBlocks;

// The reliable-update test of the iterated |r|^2 = r2 after itn
// iterations (one thread): |r| against delta times the largest |r| since
// the last update (QUDA-style reliable updates), the stop at r2stop or
// maxits, a NaN.  Returns whether the iteration goes on.  Block 0 records
// r2, rNorm, maxrr, maxrx and the pending or NaN flags.  The fields other
// blocks read are not written here (r0Norm, delta, r2stop, maxits) or are
// maxima that come out the same whether read before or after block 0's
// write (maxrr, maxrx).
__device__ __forceinline__ bool mx_test(MxState *st, double r2, int itn) {
  if (!isfinite(r2)) {
    if (blockIdx.x == 0) {
      st->r2 = r2;
      st->nan = 1;
      st->done = 1;
    }
    return false;
  }
  const double rn = sqrt(r2);
  const double maxrr = fmax(st->maxrr, rn), maxrx = fmax(st->maxrx, rn);
  const bool ux = rn < st->delta * st->r0Norm && st->r0Norm <= maxrx;
  const bool ur = (rn < st->delta * maxrr && st->r0Norm <= maxrr) || ux;
  const bool pend = ur || r2 <= st->r2stop || itn >= st->maxits;
  if (blockIdx.x == 0) {
    st->r2 = r2;
    st->rNorm = rn;
    st->maxrr = maxrr;
    st->maxrx = maxrx;
    if (pend) st->pending = 1;
  }
  return !pend;
}

// ---------------------------------------------------------------------------
// sloppy Dslash: out = b*xs + hop * sum_k [...]; fat and long partial sums
// are kept apart so that the FP16 list scales multiply them once per site.
// ---------------------------------------------------------------------------

// dslash_lo_kernel serves the FP32 links (it runs at the copy bandwidth with
// its natural registers); 16-bit links go to dslash_x2_kernel below.  The
// 16-bit kernel is instruction-heavy for the bytes it moves and gains from
// occupancy: 4 resident blocks of 64 registers (with scalar arithmetic this
// gave 4450 GB/s on 32^4 against 4090 GB/s at 72-80 registers; splitting a
// site's forward and backward hops over two threads gave 3640-3720 GB/s).

// Format of the sloppy solver's vectors p and t for a link precision: the
// same as the links.  With 16-bit links the vectors can be built in FP32
// (QS_HALF_VEC_BITS = 32); on 32^4 that keeps the iteration count (2754)
// and slows the Schur operator (90.1 against 86.2 us), so 16 is the default.
#ifndef QS_HALF_VEC_BITS
#define QS_HALF_VEC_BITS 16
#endif
template <int PREC>
struct VecPrec {
  static constexpr int v = (PREC == kF16 && QS_HALF_VEC_BITS == 32) ? kF32 : PREC;
};

struct DslashArgsLo {
  Geom g;
  int po;
  LoLinks L;
  const void *xin;
  int istride;
  const void *xs;
  int sstride;
  void *out;
  int ostride;
  float b;
  const MxState *halt;  // stop when done or pending (may be null)
  double *partials;
  unsigned *ticket;
  double *dot_out;      // RED == 2
  const float2 *rdot = nullptr;  // RED == 4, 16-bit kernel: also Re <rdot, out> partials (kMxRAp)
  // output sites [k_lo, min(k_hi, nh)) of the parity (a domain's interior or
  // its intermediate slices); site k is stored at index k - out_off of out
  int k_lo = 0, k_hi = 0x7fffffff, out_off = 0;
};

template <int PREC, int VP, int NL, int HOP, int INIT, int RED, int OUTP, int R12>
__global__ void __launch_bounds__(kBlock, PREC == kF16 ? 4 : 1) dslash_lo_kernel(const DslashArgsLo A) {
  pdl_wait();
  if (A.halt != nullptr && mx_halt(A.halt)) return;
  const Geom &g = A.g;
  const int nh = g.nh;
  const size_t V = (size_t)g.V;
  const size_t in_base = (size_t)(1 - A.po) * nh;
  const size_t out_base = (size_t)A.po * nh;
  double dot = 0.0;
  float fdot = 0.f, fdot2 = 0.f;
  const int kend = min(nh, A.k_hi);
  for (int k = A.k_lo + blockIdx.x * blockDim.x + threadIdx.x; k < kend; k += gridDim.x * blockDim.x) {
    int x[4], lex;
    site_coords(g, A.po, k, x, lex);
    float2 af[3], al[3], xsv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      af[c] = make_float2(0.f, 0.f);
      al[c] = make_float2(0.f, 0.f);
    }
    if (INIT) load_vec_cg<VP>(A.xs, A.sstride, k, xsv);
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const bool is_long = (NL == 8) && (l & 1);
      const int f = (NL == 8) ? (l >> 1) : l;
      const int jf = nbr_half(g, x, lex, mu, len);
      const int jb = nbr_half(g, x, lex, mu, -len);
      float2 v[3], w[3], uf[9], ub[9];
      load_vec<VP>(A.xin, A.istride, jf, v);
      load_vec<VP>(A.xin, A.istride, jb, w);
      if (is_long) {
        if (R12) {
          load_long12<PREC>(A.L, f, out_base + k, V, long_sign_fwd(g, x, mu), uf);
          load_long12<PREC>(A.L, f, in_base + jb, V, long_sign_bck(g, x, mu), ub);
        } else {
          load_link18<PREC>(A.L.f32_long, A.L.f32_long_tail, A.L.f16_long, A.L.f16_long_tail, f,
                            out_base + k, V, uf);
          load_link18<PREC>(A.L.f32_long, A.L.f32_long_tail, A.L.f16_long, A.L.f16_long_tail, f,
                            in_base + jb, V, ub);
        }
      } else {
        load_link18<PREC>(A.L.f32_fat, A.L.f32_fat_tail, A.L.f16_fat, A.L.f16_fat_tail, f, out_base + k,
                          V, uf);
        load_link18<PREC>(A.L.f32_fat, A.L.f32_fat_tail, A.L.f16_fat, A.L.f16_fat_tail, f, in_base + jb,
                          V, ub);
      }
      float2 t[3], q[3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        t[i] = make_float2(0.f, 0.f);
        q[i] = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          t[i] = cmadd(t[i], uf[3 * i + j], v[j]);
          q[i] = cjmadd(q[i], ub[3 * j + i], w[j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 3; i++) {
        float2 d = make_float2(t[i].x - q[i].x, t[i].y - q[i].y);
        if (is_long) {
          al[i].x += d.x;
          al[i].y += d.y;
        } else {
          af[i].x += d.x;
          af[i].y += d.y;
        }
      }
    }
    float2 o[3];
    const float sf = HOP > 0 ? A.L.fat_scale : -A.L.fat_scale;
    const float sl = HOP > 0 ? A.L.long_scale : -A.L.long_scale;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 acc = INIT ? make_float2(A.b * xsv[c].x, A.b * xsv[c].y) : make_float2(0.f, 0.f);
      acc.x = fmaf(sf, af[c].x, acc.x);
      acc.y = fmaf(sf, af[c].y, acc.y);
      if (NL == 8) {
        acc.x = fmaf(sl, al[c].x, acc.x);
        acc.y = fmaf(sl, al[c].y, acc.y);
      }
      o[c] = acc;
    }
    store_vec<OUTP>(A.out, A.ostride, k - A.out_off, o);
    if (RED == 4) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        fdot = fmaf(xsv[c].x, o[c].x, fmaf(xsv[c].y, o[c].y, fdot));
        fdot2 = fmaf(o[c].x, o[c].x, fmaf(o[c].y, o[c].y, fdot2));
      }
    } else if (RED) {
      float d = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++) d += xsv[c].x * o[c].x + xsv[c].y * o[c].y;
      dot += (double)d;
    }
  }
  if (RED == 4) {
    // per-block partials of Re <xs, out> (from 0) and |out|^2 (from kMxApAp)
    __shared__ double sh4[64];
    double v[2] = {(double)fdot, (double)fdot2};
    block_sum<2>(v, sh4);
    if (threadIdx.x == 0) {
      A.partials[blockIdx.x] = v[0];
      A.partials[kMxApAp + blockIdx.x] = v[1];
    }
  } else if (RED == 2) {
    double v[1] = {dot}, s[1];
    if (grid_reduce<1>(v, A.partials, A.ticket, s) && threadIdx.x == 0) *A.dot_out = s[0];
  }
}

// The 16-bit half sweep in packed FP32x2 arithmetic.  Per site and hop:
//   forward  t_i = sum_j U_ij(x) v_j,             v = xin(x + d)
//   backward q_i = sum_j conj(U_ji(x - d)) w_j,   w = xin(x - d)
// accumulated as d = sum (t - q) = T + i S with T = sum (u Re v), S =
// sum (u Im v) over (re, im) pairs u of the links: the backward link is
// decoded directly as -conj(U) (its row 2 rebuilt with -k) so that its
// terms add.  The long hops' vectors are scaled by long_scale / fat_scale,
// so one set of accumulators carries both lists in fat units.
template <int VP, int NL, int HOP, int INIT, int RED, int OUTP, int R12>
__global__ void __launch_bounds__(kBlock, 4) dslash_x2_kernel(const DslashArgsLo A) {
  pdl_wait();
  if (A.halt != nullptr && mx_halt(A.halt)) return;
  const Geom &g = A.g;
  const int nh = g.nh;
  const size_t V = (size_t)g.V;
  const size_t in_base = (size_t)(1 - A.po) * nh;
  const size_t out_base = (size_t)A.po * nh;
  const float rho = A.L.long_scale / A.L.fat_scale;
  double dot = 0.0;
  float fdot = 0.f, fdot2 = 0.f, fdot3 = 0.f;
  const int kend = min(nh, A.k_hi);
  for (int k = A.k_lo + blockIdx.x * blockDim.x + threadIdx.x; k < kend; k += gridDim.x * blockDim.x) {
    int x[4], lex;
    site_coords(g, A.po, k, x, lex);
    float2 T[3], S[3], xsv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      T[c] = make_float2(0.f, 0.f);
      S[c] = make_float2(0.f, 0.f);
    }
    if (INIT) load_vec_cg<VP>(A.xs, A.sstride, k, xsv);
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const bool is_long = (NL == 8) && (l & 1);
      const int f = (NL == 8) ? (l >> 1) : l;
      const int jf = nbr_half(g, x, lex, mu, len);
      const int jb = nbr_half(g, x, lex, mu, -len);
      const float s = is_long ? rho : 1.f;
      float2 br[3], bi[3], u[9];
      // forward hop
      load_vec_bc<VP>(A.xin, A.istride, jf, s, br, bi);
      if (is_long) {
        if (R12)
          load_long12_x2<1, 1>(A.L, f, out_base + k, V, long_sign_fwd(g, x, mu) * A.L.long_rc, u);
        else
          load_link18_x2<1, 1>(A.L.f16_long, A.L.f16_long_tail, f, out_base + k, V, u);
      } else {
        load_link18_x2<1, 1>(A.L.f16_fat, A.L.f16_fat_tail, f, out_base + k, V, u);
      }
#pragma unroll
      for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
          T[i] = __ffma2_rn(u[3 * i + j], br[j], T[i]);
          S[i] = __ffma2_rn(u[3 * i + j], bi[j], S[i]);
        }
      }
      // backward hop, link decoded as -conj(U)
      load_vec_bc<VP>(A.xin, A.istride, jb, s, br, bi);
      if (is_long) {
        if (R12)
          load_long12_x2<-1, 1>(A.L, f, in_base + jb, V, -long_sign_bck(g, x, mu) * A.L.long_rc, u);
        else
          load_link18_x2<-1, 1>(A.L.f16_long, A.L.f16_long_tail, f, in_base + jb, V, u);
      } else {
        load_link18_x2<-1, 1>(A.L.f16_fat, A.L.f16_fat_tail, f, in_base + jb, V, u);
      }
#pragma unroll
      for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
          T[i] = __ffma2_rn(u[3 * j + i], br[j], T[i]);
          S[i] = __ffma2_rn(u[3 * j + i], bi[j], S[i]);
        }
      }
    }
    float2 o[3];
    const float sf = HOP > 0 ? A.L.fat_scale : -A.L.fat_scale;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 d = make_float2(T[c].x - S[c].y, T[c].y + S[c].x);
      float2 acc = INIT ? make_float2(A.b * xsv[c].x, A.b * xsv[c].y) : make_float2(0.f, 0.f);
      acc.x = fmaf(sf, d.x, acc.x);
      acc.y = fmaf(sf, d.y, acc.y);
      o[c] = acc;
    }
    store_vec<OUTP>(A.out, A.ostride, k - A.out_off, o);
    if (RED == 4) {
      // FP32 per thread (a thread holds one or two sites): two registers
      // fewer than FP64 sums, which the 64-register budget needs
#pragma unroll
      for (int c = 0; c < 3; c++) {
        fdot = fmaf(xsv[c].x, o[c].x, fmaf(xsv[c].y, o[c].y, fdot));
        fdot2 = fmaf(o[c].x, o[c].x, fmaf(o[c].y, o[c].y, fdot2));
      }
      if (A.rdot != nullptr) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float2 r = __ldcg(A.rdot + (size_t)c * A.ostride + (k - A.out_off));
          fdot3 = fmaf(r.x, o[c].x, fmaf(r.y, o[c].y, fdot3));
        }
      }
    } else if (RED) {
      float dd = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++) dd += xsv[c].x * o[c].x + xsv[c].y * o[c].y;
      dot += (double)dd;
    }
  }
  if (RED == 4) {
    __shared__ double sh4[96];
    double v[3] = {(double)fdot, (double)fdot2, (double)fdot3};
    block_sum<3>(v, sh4);
    if (threadIdx.x == 0) {
      A.partials[blockIdx.x] = v[0];
      A.partials[kMxApAp + blockIdx.x] = v[1];
      if (A.rdot != nullptr) A.partials[kMxRAp + blockIdx.x] = v[2];
    }
  } else if (RED == 2) {
    double v[1] = {dot}, sm[1];
    if (grid_reduce<1>(v, A.partials, A.ticket, sm) && threadIdx.x == 0) *A.dot_out = sm[0];
  }
}

// Grid of a sloppy half sweep.  The 16-bit kernel runs exactly two waves of
// resident blocks (occupancy from the runtime, so that no partial wave idles
// SMs: on 32^4 two waves gave 5208 GB/s, 1.5 waves 4437); the FP32 kernel is
// at the copy bandwidth with 4 blocks per SM.
template <int PREC, int VP, int NL, int HOP, int INIT, int RED, int OUTP, int R12>
static int lo_grid(int nh) {
  static int resident = 0;  // one per kernel instantiation
  if (resident == 0) {
    int n = 0;
    cudaError_t e;
    if constexpr (PREC == kF16)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dslash_x2_kernel<VP, NL, HOP, INIT, RED, OUTP, R12>,
                                                        kBlock, 0);
    else
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dslash_lo_kernel<PREC, VP, NL, HOP, INIT, RED, OUTP, R12>,
                                                        kBlock, 0);
    if (e != cudaSuccess || n < 1) {
      cudaGetLastError();
      n = 4;
    }
    resident = n;
  }
  long want = (long)num_sms() * (PREC == kF16 ? 2 * resident : 4);
  long need = (nh + kBlock - 1) / kBlock;
  long g = want < need ? want : need;
  if (g > kMaxRedBlocks) g = kMaxRedBlocks;
  return (int)(g < 1 ? 1 : g);
}

// returns the grid launched
template <int PREC, int VP, int NL, int HOP, int INIT, int RED, int OUTP>
static int launch_lo(const DslashArgsLo &A, int) {
  int grid;
  const int nsites = std::max(0, std::min(A.g.nh, A.k_hi) - A.k_lo);
  if constexpr (PREC == kF16) {
    if (NL == 8 && A.L.recon12) {
      grid = lo_grid<PREC, VP, NL, HOP, INIT, RED, OUTP, 1>(nsites);
      launch_pdl(dslash_x2_kernel<VP, NL, HOP, INIT, RED, OUTP, 1>, grid, kBlock, A);
    } else {
      grid = lo_grid<PREC, VP, NL, HOP, INIT, RED, OUTP, 0>(nsites);
      launch_pdl(dslash_x2_kernel<VP, NL, HOP, INIT, RED, OUTP, 0>, grid, kBlock, A);
    }
  } else if (NL == 8 && A.L.recon12) {
    grid = lo_grid<PREC, VP, NL, HOP, INIT, RED, OUTP, 1>(nsites);
    launch_pdl(dslash_lo_kernel<PREC, VP, NL, HOP, INIT, RED, OUTP, 1>, grid, kBlock, A);
  } else {
    grid = lo_grid<PREC, VP, NL, HOP, INIT, RED, OUTP, 0>(nsites);
    launch_pdl(dslash_lo_kernel<PREC, VP, NL, HOP, INIT, RED, OUTP, 0>, grid, kBlock, A);
  }
  note_launch();
  return grid;
}

// the two half sweeps of the sloppy Schur operator:
//   which 0: t = (2D)_{q,par} p                (out: PREC, hop +1)
//   which 1: ap = 4 m2 p - (2D)_{par,q} t      (out: FP32, hop -1, pAp)
//   red 2: Re <p, Ap> summed into *dot_out (last-block reduction)
//   red 4: per-block partials of <p, Ap> in partials[0 .. *blocks) and of
//          |Ap|^2 from partials[kMxApAp]; with A.rdot (16-bit links) also
//          of Re <rdot, Ap> from partials[kMxRAp]
template <int PREC, int NL>
static int sloppy_half(int which, const DslashArgsLo &A, int grid, int red, int *blocks) {
  constexpr int VP = VecPrec<PREC>::v;
  int used;
  if (which == 0) {
    used = launch_lo<PREC, VP, NL, 1, 0, 0, VP>(A, grid);
  } else if (red == 2) {
    used = launch_lo<PREC, VP, NL, -1, 1, 2, kF32>(A, grid);
  } else if (red == 4) {
    used = launch_lo<PREC, VP, NL, -1, 1, 4, kF32>(A, grid);
  } else {
    used = launch_lo<PREC, VP, NL, -1, 1, 0, kF32>(A, grid);
  }
  if (blocks) *blocks = used;
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// sloppy Schur: ap (FP32 [3][nh]) = 4 m2 p - (2D)(2D) p on parity par,
// p and t in format prec; rdot (FP32 [3][nh], 16-bit links and red 4 only)
// adds the Re <rdot, ap> partials.
int schur_lo(const qexstag_links_s *g, int prec, int par, float2 *ap, const void *p, void *t,
             double m2, int red, const MxState *halt, double *dot_out, int *red_blocks,
             const float2 *rdot = nullptr) {
  const Geom &geo = g->l->g;
  DslashArgsLo A;
  A.g = geo;
  A.L = lo_links(g->low, prec);
  A.halt = halt;
  A.partials = red_partials();
  A.ticket = red_tickets();
  A.dot_out = dot_out;
  const int grid = 0;  // chosen per kernel by launch_lo
  // half sweep 1
  A.po = 1 - par;
  A.xin = p;
  A.istride = geo.nh;
  A.xs = nullptr;
  A.sstride = 0;
  A.out = t;
  A.ostride = geo.nh;
  A.b = 0.f;
  int rc;
  if (prec == kF32)
    rc = g->nl == 8 ? sloppy_half<kF32, 8>(0, A, grid, 0, nullptr) : sloppy_half<kF32, 4>(0, A, grid, 0, nullptr);
  else
    rc = g->nl == 8 ? sloppy_half<kF16, 8>(0, A, grid, 0, nullptr) : sloppy_half<kF16, 4>(0, A, grid, 0, nullptr);
  if (rc) return rc;
  // half sweep 2
  A.po = par;
  A.xin = t;
  A.xs = p;
  A.sstride = geo.nh;
  A.out = ap;
  A.b = (float)(4.0 * m2);
  A.rdot = rdot;
  if (prec == kF32)
    rc = g->nl == 8 ? sloppy_half<kF32, 8>(1, A, grid, red, red_blocks)
                    : sloppy_half<kF32, 4>(1, A, grid, red, red_blocks);
  else
    rc = g->nl == 8 ? sloppy_half<kF16, 8>(1, A, grid, red, red_blocks)
                    : sloppy_half<kF16, 4>(1, A, grid, red, red_blocks);
  return rc;
}

// sloppy Schur with FP32 vectors whatever the link precision (the
// single-right-hand-side multi-shift CG): ap = 4 m2 p - (2D)(2D) p on parity
// par, t the FP32 temporary, *dot_out = Re <p, ap> (FP64 sum)
int schur_lo_v32(const qexstag_links_s *g, int prec, int par, float2 *ap, const float2 *p, float2 *t, double m2,
                 double *dot_out) {
  const Geom &geo = g->l->g;
  DslashArgsLo A;
  A.g = geo;
  A.L = lo_links(g->low, prec);
  A.halt = nullptr;
  A.partials = red_partials();
  A.ticket = red_tickets();
  A.dot_out = dot_out;
  A.po = 1 - par;
  A.xin = p;
  A.istride = geo.nh;
  A.xs = nullptr;
  A.sstride = 0;
  A.out = t;
  A.ostride = geo.nh;
  A.b = 0.f;
  auto sweeps = [&](auto nl) {
    constexpr int NL = decltype(nl)::value;
    if (prec == kF16)
      launch_lo<kF16, kF32, NL, 1, 0, 0, kF32>(A, 0);
    else
      launch_lo<kF32, kF32, NL, 1, 0, 0, kF32>(A, 0);
    A.po = par;
    A.xin = t;
    A.xs = p;
    A.sstride = geo.nh;
    A.out = ap;
    A.b = (float)(4.0 * m2);
    if (prec == kF16)
      launch_lo<kF16, kF32, NL, -1, 1, 2, kF32>(A, 0);
    else
      launch_lo<kF32, kF32, NL, -1, 1, 2, kF32>(A, 0);
  };
  if (g->nl == 8)
    sweeps(std::integral_constant<int, 8>());
  else
    sweeps(std::integral_constant<int, 4>());
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// mixed CG kernels
// ---------------------------------------------------------------------------

template <int PREC>
__global__ void __launch_bounds__(kBlock)
    mx_init_kernel(const double2 *__restrict__ b, int bs, double2 *__restrict__ x, double2 *__restrict__ r,
                   float2 *__restrict__ rs, float2 *__restrict__ xs, void *p, int n, MxState *st,
                   double *partials, unsigned *ticket) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 pv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 v = b[(size_t)c * bs + i];
      x[(size_t)c * n + i] = make_double2(0.0, 0.0);
      r[(size_t)c * n + i] = v;
      pv[c] = make_float2((float)v.x, (float)v.y);
      rs[(size_t)c * n + i] = pv[c];
      xs[(size_t)c * n + i] = make_float2(0.f, 0.f);
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
    store_vec<PREC>(p, n, i, pv);
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) {
    double b2 = o[0];
    st->b2 = b2;
    st->r2 = b2;
    st->r2old = b2;
    st->r2stop = st->r2req * b2;
    st->rNorm = st->r0Norm = st->maxrx = st->maxrr = sqrt(b2);
    st->itn = 0;
    st->pending = 0;
    st->reliable = 0;
    st->nan = isfinite(b2) ? 0 : 1;
    st->done = (!(b2 > st->r2stop) || st->maxits <= 0 || st->nan) ? 1 : 0;
  }
}

// The fused update of the three-kernel iteration (iteration k + 1):
//   the reliable-update test of |r_{k+1}|^2 (the previous update's per-block
//   partials at r2in, nr2 of them; nr2 = 0 right after the start or a
//   reliable update, when r2 is the state's), then
//   rs -= alpha ap; xs += alpha p_in; p_out = rs + beta p_in
// with alpha = r2 / <p, Ap> and beta from the half sweep's per-block
// partials (np of each): with the partials of Re <r, Ap> (rap: the 16-bit
// solves, on one lattice or a domain), beta = -<r_new, Ap> / <p, Ap> = (alpha |Ap|^2 -
// <r, Ap>) / <p, Ap>, the beta that makes the next direction A-orthogonal
// to p for the operator actually applied; without them (rap null) beta =
// (alpha^2 |Ap|^2 - r2) / r2, the same value once <r, Ap> = <p, Ap>.  In
// exact arithmetic both are CG's |r_new|^2 / |r|^2 (cg.nim:229-236),
// through |r - alpha Ap|^2 = r2 - 2 alpha <r, Ap> + alpha^2 |Ap|^2 and
// <r, Ap> = <p, Ap>.  With 16-bit links the first form took 2828
// iterations at 32^4 and delta 0.1 where the second took 2880.  Every block
// adds each set of partials in the same order, so all take the same
// decisions.  So p needs no second pass over the sites; the exact
// |r_new|^2 is summed as well (per-block partials at r2out) for the next
// update's alpha and test.  When the test stops the iteration nothing is
// written: p_in, the direction a reliable update corrects, is intact in its
// buffer (p_out is the other one), and the half sweeps of this iteration
// were spent for nothing (once per reliable update).  Block 0 records the
// state; the iteration count the blocks test is itc[par], and block 0 writes
// itc[par ^ 1] (the host alternates par; a reliable update sets both).
template <int PREC>
__global__ void __launch_bounds__(kBlock)
    mx_update_p_kernel(float2 *__restrict__ rs, float2 *__restrict__ xs, const float2 *__restrict__ ap,
                       const void *pin, void *pout, int n, MxState *st, const double *pap, const double *apap,
                       int np, const double *r2in, int nr2, double *r2out, int par, const double *rap = nullptr) {
  pdl_wait();
  if (mx_halt(st)) return;
  // the first site's operands are loaded before the sums of the partials,
  // so that their latencies overlap
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  float2 pv[3], rv[3], av[3], xv[3];
  if (i0 < n) {
    load_vec<PREC>(pin, n, i0, pv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      rv[c] = rs[(size_t)c * n + i0];
      av[c] = ap[(size_t)c * n + i0];
      xv[c] = xs[(size_t)c * n + i0];
    }
  }
  // the partials, summed by the whole block (one round of loads)
  __shared__ float sh_ab[2];
  __shared__ int sh_go;
  {
    double v3[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
      v3[0] += __ldcg(pap + i);
      v3[1] += __ldcg(apap + i);
      if (rap != nullptr) v3[3] += __ldcg(rap + i);
    }
    for (int i = threadIdx.x; i < nr2; i += blockDim.x) v3[2] += __ldcg(r2in + i);
    __shared__ double shp[128];
    block_sum<4>(v3, shp);
    if (threadIdx.x == 0) {
      const double s = v3[0], q = v3[1];
      const int itn = st->itc[par];
      double r2 = st->r2;
      bool go = true;
      if (nr2 > 0) {
        r2 = v3[2];
        go = mx_test(st, r2, itn);
      }
      if (go) {
        const double alpha = r2 / s;
        const double beta = rap != nullptr ? (alpha * q - v3[3]) / s : (alpha * alpha * q - r2) / r2;
        sh_ab[0] = (float)alpha;
        sh_ab[1] = (float)beta;
        if (blockIdx.x == 0) {
          st->pAp = s;
          st->alpha = alpha;
          st->beta = beta;
          st->itn = itn + 1;
          st->itc[par ^ 1] = itn + 1;
          st->r2old = r2;
          st->pin = par;
        }
      }
      sh_go = go ? 1 : 0;
    }
  }
  __syncthreads();
  if (!sh_go) return;
  const float alpha = sh_ab[0], beta = sh_ab[1];
  double s = 0.0;
  for (int i = i0; i < n; i += gridDim.x * blockDim.x) {
    if (i != i0) {
      load_vec<PREC>(pin, n, i, pv);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        rv[c] = rs[(size_t)c * n + i];
        av[c] = ap[(size_t)c * n + i];
        xv[c] = xs[(size_t)c * n + i];
      }
    }
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 r = rv[c], x = xv[c];
      r.x = fmaf(-alpha, av[c].x, r.x);
      r.y = fmaf(-alpha, av[c].y, r.y);
      x.x = fmaf(alpha, pv[c].x, x.x);
      x.y = fmaf(alpha, pv[c].y, x.y);
      rs[(size_t)c * n + i] = r;
      xs[(size_t)c * n + i] = x;
      acc = fmaf(r.x, r.x, acc);
      acc = fmaf(r.y, r.y, acc);
      pv[c] = make_float2(fmaf(beta, pv[c].x, r.x), fmaf(beta, pv[c].y, r.y));
    }
    store_vec<PREC>(pout, n, i, pv);
    s += (double)acc;
  }
  __shared__ double sh[32];
  double v[1] = {s};
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) r2out[blockIdx.x] = v[0];
}

// reliable update part 1: x += xs, xs = 0
__global__ void mx_flush_kernel(double2 *__restrict__ x, float2 *__restrict__ xs, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) {
    float2 v = xs[i];
    double2 w = x[i];
    w.x += (double)v.x;
    w.y += (double)v.y;
    x[i] = w;
    xs[i] = make_float2(0.f, 0.f);
  }
}

// reliable update part 2: r = b - Ax (FP64), rs = r, true |r|^2 and decisions
__global__ void __launch_bounds__(kBlock)
    mx_true_res_kernel(const double2 *__restrict__ b, int bs, const double2 *__restrict__ ax,
                       double2 *__restrict__ r, float2 *__restrict__ rs, int n, MxState *st,
                       double *partials, unsigned *ticket) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 bv = b[(size_t)c * bs + i], a = ax[(size_t)c * n + i];
      double2 v = make_double2(bv.x - a.x, bv.y - a.y);
      r[(size_t)c * n + i] = v;
      rs[(size_t)c * n + i] = make_float2((float)v.x, (float)v.y);
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) {
    const double r2 = o[0];
    st->r2 = r2;
    st->reliable += 1;
    if (!isfinite(r2)) {
      st->nan = 1;
      st->done = 1;
      return;
    }
    if (r2 <= st->r2stop || st->itn >= st->maxits) {
      st->done = 1;
      return;
    }
    const double rn = sqrt(r2);
    st->rNorm = st->r0Norm = st->maxrr = st->maxrx = rn;
    st->beta = r2 / st->r2old;
    st->itc[0] = st->itc[1] = st->itn;
  }
}

// reliable update part 3: rp = <rs, p>
template <int PREC>
__global__ void __launch_bounds__(kBlock)
    mx_rp_kernel(const float2 *__restrict__ rs, const void *p, int n, MxState *st, double *partials,
                 unsigned *ticket) {
  if (st->done) return;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 pv[3];
    load_vec<PREC>(p, n, i, pv);
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 r = rs[(size_t)c * n + i];
      acc = fmaf(r.x, pv[c].x, acc);
      acc = fmaf(r.y, pv[c].y, acc);
    }
    s += (double)acc;
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) st->rp = o[0];
}

// reliable update part 4: p = rs + beta (p - (rp/r2) rs); clears pending
template <int PREC>
__global__ void mx_p_reliable_kernel(const float2 *__restrict__ rs, void *p, int n, MxState *st) {
  if (st->done) return;
  const float beta = (float)st->beta;
  const float g = (float)(st->rp / st->r2);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 pv[3];
    load_vec_cg<PREC>(p, n, i, pv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 r = rs[(size_t)c * n + i];
      float2 q = make_float2(fmaf(-g, r.x, pv[c].x), fmaf(-g, r.y, pv[c].y));
      pv[c] = make_float2(fmaf(beta, q.x, r.x), fmaf(beta, q.y, r.y));
    }
    store_vec<PREC>(p, n, i, pv);
  }
}

__global__ void mx_clear_pending_kernel(MxState *st) { st->pending = 0; }

static_assert(sizeof(MxState) <= sizeof(double) * kNumResults, "state too large for the staging buffer");

int check_interval(int nh);

template <int PREC>
static int cg_mixed_t(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req,
                      int maxits, double delta, CgOut *out, int *reliable) {
  constexpr int VP = VecPrec<PREC>::v;  // format of p and t
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  Workspace &ws = g->ws;
  const size_t v64 = sizeof(double2) * 3 * (size_t)nh, v32 = sizeof(float2) * 3 * (size_t)nh;
  const size_t vp = (VP == kF32) ? v32 : sizeof(uint4) * (size_t)nh;
  void *pr, *pax, *prs, *pxs, *pap, *pp, *pp2, *pt, *pt64, *pst;
  int rc;
  if ((rc = ws.get(kSlotMx0 + 0, v64, &pr)) || (rc = ws.get(kSlotMx0 + 1, v64, &pax)) ||
      (rc = ws.get(kSlotMx0 + 2, v32, &prs)) || (rc = ws.get(kSlotMx0 + 3, v32, &pxs)) ||
      (rc = ws.get(kSlotMx0 + 4, v32, &pap)) || (rc = ws.get(kSlotMx0 + 5 + 2 * VP, vp, &pp)) ||
      (rc = ws.get(kSlotMx0 + 6 + 2 * VP, vp, &pt)) || (rc = ws.get(kSlotMx0 + 9, v64, &pt64)) ||
      (rc = ws.get(kSlotMx0 + 10, sizeof(MxState), &pst)) || (rc = ws.get(kSlotMx0 + 12 + VP, vp, &pp2)))
    return rc;
  // p alternates between two buffers: each fused update reads one and
  // writes the other
  void *const P[2] = {pp, pp2};
  double2 *r = (double2 *)pr, *ax = (double2 *)pax;
  float2 *rs = (float2 *)prs, *xs = (float2 *)pxs, *ap = (float2 *)pap;
  MxState *st = (MxState *)pst;
  MxState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.r2req = r2req;
  hs.maxits = maxits;
  hs.delta = delta;
  {
    double *buf = host_results();
    std::memcpy(buf, &hs, sizeof(hs));
    QS_CUDA(cudaMemcpyAsync(st, buf, sizeof(hs), cudaMemcpyHostToDevice, stream()));
  }
  const int grid = grid_for(nh, kBlock, 4);
  const int egrid = grid_for(nh, kBlock, 8);
  mx_init_kernel<VP><<<grid, kBlock, 0, stream()>>>(b.p, b.stride, x.p, r, rs, xs, pp, nh, st,
                                                      red_partials(), red_tickets());
  note_launch();
  QS_LAUNCH_CHECK();
  const int every = check_interval(nh);
  // Three kernels an iteration: the two half sweeps (the second leaves the
  // <p, Ap> and |Ap|^2 partials) and the fused update, which first tests the
  // previous update's |r|^2 (except right after the start or a reliable
  // update).  cur: the host parity of the next iteration, which reads p from
  // P[cur] and |r|^2 partials from R2[cur], and writes P[cur ^ 1], R2[cur ^ 1].
  int cur = 0;
  bool fresh = true;
  double *const R2[2] = {red_partials() + kMxR2, red_partials() + kMxR2b};
  auto batch = [&]() -> int {
    for (int i = 0; i < every; i++) {
      int np = 0;
      constexpr bool hs = PREC == kF16;  // <r, Ap> partials from half sweep 2
      int rc2 = schur_lo(g, PREC, par, ap, P[cur], pt, m2, 4, st, nullptr, &np, hs ? rs : nullptr);
      if (rc2) return rc2;
      launch_pdl(mx_update_p_kernel<VP>, grid, kBlock, rs, xs, (const float2 *)ap, (const void *)P[cur],
                 P[cur ^ 1], nh, st, (const double *)red_partials(), (const double *)(red_partials() + kMxApAp),
                 np, (const double *)R2[cur], fresh ? 0 : grid, R2[cur ^ 1], cur,
                 hs ? (const double *)(red_partials() + kMxRAp) : (const double *)nullptr);
      note_launch();
      cur ^= 1;
      fresh = false;
    }
    QS_LAUNCH_CHECK();
    return QEXSTAG_OK;
  };
  // The state is read one batch behind: the next batch is queued before the
  // host waits for the snapshot.  When the snapshot shows the solve done or
  // a reliable update due, that batch's kernels have returned at once
  // (done / pending), and the update is queued after them.
  StateSnapshot snap;
  if ((rc = batch())) return rc;
  for (;;) {
    if ((rc = snap.start(st, sizeof(MxState))) || (rc = batch()) || (rc = snap.wait(&hs, sizeof(MxState))))
      return rc;
    if (hs.done) break;
    if (!hs.pending) continue;
    // reliable update: fold the increment in, FP64 true residual; the
    // direction corrected is the one the last update that ran read
    // (P[hs.pin]: the update that stopped wrote nothing, and the kernels
    // queued after it returned at once), and the iteration goes on from it
    mx_flush_kernel<<<egrid, kBlock, 0, stream()>>>(x.p, xs, nh);
    note_launch();
    if ((rc = schur64(g, par, VecD{ax, nh}, cv(x), VecD{(double2 *)pt64, nh}, m2))) return rc;
    cur = hs.pin & 1;
    fresh = true;
    mx_true_res_kernel<<<grid, kBlock, 0, stream()>>>(b.p, b.stride, ax, r, rs, nh, st, red_partials(),
                                                      red_tickets());
    mx_rp_kernel<VP><<<grid, kBlock, 0, stream()>>>(rs, P[cur], nh, st, red_partials(), red_tickets());
    mx_p_reliable_kernel<VP><<<egrid, kBlock, 0, stream()>>>(rs, P[cur], nh, st);
    mx_clear_pending_kernel<<<1, 1, 0, stream()>>>(st);
    note_launch(4);
    QS_LAUNCH_CHECK();
    if ((rc = batch())) return rc;
  }
  out->iterations = hs.itn;
  out->r2 = hs.b2 > 0 ? hs.r2 / hs.b2 : 0.0;
  out->nan = hs.nan;
  *reliable = hs.reliable;
  if (hs.nan) return fail(QEXSTAG_ERR_NAN, "mixed cg: NaN in residual");
  return QEXSTAG_OK;
}

int cg_mixed(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits,
             int sloppy, double delta, CgOut *out, int *reliable) {
  if (!g->low.ready) return fail(QEXSTAG_ERR_STATE, "reduced-precision links missing");
  if (x.stride != g->l->g.V && x.stride != g->l->g.nh)
    return fail(QEXSTAG_ERR_ARG, "cg_mixed: bad solution stride");
  // the solution accumulates in a compact [3][nh] buffer, copied out at the end
  const int nh = g->l->g.nh;
  void *px;
  int rc = g->ws.get(kSlotMx0 + 11, sizeof(double2) * 3 * (size_t)nh, &px);
  if (rc) return rc;
  VecD xc{(double2 *)px, nh};
  rc = (sloppy == QEXSTAG_SLOPPY_HALF) ? cg_mixed_t<kF16>(g, par, m2, b, xc, r2req, maxits, delta, out, reliable)
                                       : cg_mixed_t<kF32>(g, par, m2, b, xc, r2req, maxits, delta, out, reliable);
  if (rc) return rc;
  return vcopy(x, cv(xc), nh);
}

// ---------------------------------------------------------------------------
// the 16-bit reliable-update CG on one domain of a decomposed lattice
//
// The same iteration as cg_mixed_t on the domain's extended lattice: half
// sweep 1 on the odd slices the second needs ([odd_lo, odd_hi), reaching
// rho slices into the ghosts), half sweep 2 and the vector updates on the
// interior even sites.  Before half sweep 1 the ghost slices of p (16 bytes
// per site) are exchanged, and every sum (<p, Ap>, |Ap|^2 and |r|^2 once per
// iteration, and at reliable updates |b - Ax|^2 and <r, p>) is the domain's
// partial, added in block order, then summed over the processes, before the
// state kernels use it.
// The caller provides the exchange, the sum and the FP64 Schur operator of
// the decomposed lattice (MxDomain).
// ---------------------------------------------------------------------------

// sum of np partials into *val (one block, fixed order)
__global__ void mxd_sum_kernel(const double *partials, int np, double *val) {
  __shared__ double sh[32];
  double v[1] = {0.0};
  for (int i = threadIdx.x; i < np; i += blockDim.x) v[0] += __ldcg(partials + i);
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) *val = v[0];
}

// the four sums of an iteration, in block order: <p, Ap>, |Ap|^2 and
// Re <r, Ap> (np half-sweep partials each) and the previous update's |r|^2
// (nr2 partials, 0 when there is none) into val[0..3] as <p, Ap>, |Ap|^2,
// |r|^2, <r, Ap>
__global__ void mxd_sum4_kernel(const double *pap, const double *apap, const double *rap, int np,
                                const double *r2p, int nr2, double *val) {
  __shared__ double sh[128];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    v[0] += __ldcg(pap + i);
    v[1] += __ldcg(apap + i);
    v[3] += __ldcg(rap + i);
  }
  for (int i = threadIdx.x; i < nr2; i += blockDim.x) v[2] += __ldcg(r2p + i);
  block_sum<4>(v, sh);
  if (threadIdx.x == 0) {
    val[0] = v[0];
    val[1] = v[1];
    val[2] = v[2];
    val[3] = v[3];
  }
}

// r = b, x = 0, rs = b, xs = 0, p = b; per-block |b|^2
template <int VP>
__global__ void __launch_bounds__(kBlock)
    mxd_init_kernel(const double2 *__restrict__ b, double2 *__restrict__ x, double2 *__restrict__ r,
                    float2 *__restrict__ rs, float2 *__restrict__ xs, void *p, int n, double *partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 pv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 v = b[(size_t)c * n + i];
      x[(size_t)c * n + i] = make_double2(0.0, 0.0);
      r[(size_t)c * n + i] = v;
      pv[c] = make_float2((float)v.x, (float)v.y);
      rs[(size_t)c * n + i] = pv[c];
      xs[(size_t)c * n + i] = make_float2(0.f, 0.f);
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
    store_vec<VP>(p, n, i, pv);
  }
  __shared__ double sh[32];
  double v[1] = {s};
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// the state at the start (as mx_init_kernel), from the summed |b|^2
__global__ void mxd_init_state_kernel(MxState *st, const double *b2p) {
  const double b2 = *b2p;
  st->b2 = b2;
  st->r2 = b2;
  st->r2old = b2;
  st->r2stop = st->r2req * b2;
  st->rNorm = st->r0Norm = st->maxrx = st->maxrr = sqrt(b2);
  st->itn = 0;
  st->itc[0] = st->itc[1] = 0;
  st->pending = 0;
  st->reliable = 0;
  st->nan = isfinite(b2) ? 0 : 1;
  st->done = (!(b2 > st->r2stop) || st->maxits <= 0 || st->nan) ? 1 : 0;
}

// reliable update: r = b - Ax, rs = r; per-block |r|^2
__global__ void __launch_bounds__(kBlock)
    mxd_true_res_kernel(const double2 *__restrict__ b, const double2 *__restrict__ ax, double2 *__restrict__ r,
                        float2 *__restrict__ rs, int n, double *partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 bv = b[(size_t)c * n + i], a = ax[(size_t)c * n + i];
      const double2 v = make_double2(bv.x - a.x, bv.y - a.y);
      r[(size_t)c * n + i] = v;
      rs[(size_t)c * n + i] = make_float2((float)v.x, (float)v.y);
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
  }
  __shared__ double sh[32];
  double v[1] = {s};
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// the decisions of mx_true_res_kernel from the summed true |r|^2
__global__ void mxd_true_res_state_kernel(MxState *st, const double *r2p) {
  const double r2 = *r2p;
  st->r2 = r2;
  st->reliable += 1;
  if (!isfinite(r2)) {
    st->nan = 1;
    st->done = 1;
    return;
  }
  if (r2 <= st->r2stop || st->itn >= st->maxits) {
    st->done = 1;
    return;
  }
  const double rn = sqrt(r2);
  st->rNorm = st->r0Norm = st->maxrr = st->maxrx = rn;
  st->beta = r2 / st->r2old;
  st->itc[0] = st->itc[1] = st->itn;
}

// per-block <rs, p> (mx_rp_kernel without the grid reduction)
template <int PREC>
__global__ void __launch_bounds__(kBlock)
    mxd_rp_kernel(const float2 *__restrict__ rs, const void *p, int n, double *partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 pv[3];
    load_vec<PREC>(p, n, i, pv);
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 r = rs[(size_t)c * n + i];
      acc = fmaf(r.x, pv[c].x, acc);
      acc = fmaf(r.y, pv[c].y, acc);
    }
    s += (double)acc;
  }
  __shared__ double sh[32];
  double v[1] = {s};
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

__global__ void mxd_set_rp_kernel(MxState *st, const double *rp) {
  if (!st->done) st->rp = *rp;
}

int cg_mixed_domain(const MxDomain &D, double m2, const double2 *b, double2 *x, double r2req, int maxits,
                    double delta, CgOut *out, int *reliable) {
  constexpr int PREC = kF16;
  constexpr int VP = VecPrec<PREC>::v;
  static_assert(VP == kF16, "the ghost exchange moves 16-byte sites");
  qexstag_links_s *g = D.g;
  if (!g->low.ready) return fail(QEXSTAG_ERR_STATE, "domain mixed cg: reduced-precision links missing");
  const Geom &geo = g->l->g;
  const int n = D.n, nh = geo.nh;
  Workspace &ws = g->ws;
  const size_t v64 = sizeof(double2) * 3 * (size_t)n, v32 = sizeof(float2) * 3 * (size_t)n;
  void *pr, *pax, *prs, *pxs, *pap, *pp, *pp2, *pt, *pst, *pval, *ppart;
  int rc;
  if ((rc = ws.get(kSlotMx0 + 30, v64, &pr)) || (rc = ws.get(kSlotMx0 + 31, v64, &pax)) ||
      (rc = ws.get(kSlotMx0 + 32, v32, &prs)) || (rc = ws.get(kSlotMx0 + 33, v32, &pxs)) ||
      (rc = ws.get(kSlotMx0 + 34, v32, &pap)) || (rc = ws.get(kSlotMx0 + 35, sizeof(uint4) * (size_t)nh, &pp)) ||
      (rc = ws.get(kSlotMx0 + 36, sizeof(uint4) * (size_t)nh, &pt)) ||
      (rc = ws.get(kSlotMx0 + 37, sizeof(MxState), &pst)) || (rc = ws.get(kSlotMx0 + 38, sizeof(double) * 4, &pval)) ||
      (rc = ws.get(kSlotMx0 + 39, sizeof(double) * 5 * kMaxRedBlocks, &ppart)) ||
      (rc = ws.get(kSlotMx0 + 40, sizeof(uint4) * (size_t)nh, &pp2)))
    return rc;
  double2 *r = (double2 *)pr, *ax = (double2 *)pax;
  float2 *rs = (float2 *)prs, *xs = (float2 *)pxs, *ap = (float2 *)pap;
  uint4 *t = (uint4 *)pt;
  // p alternates between two extended-lattice buffers (the fused update
  // reads one and writes the other); PI: their interior parts, compact
  uint4 *const P[2] = {(uint4 *)pp, (uint4 *)pp2};
  uint4 *const PI[2] = {P[0] + D.even_lo, P[1] + D.even_lo};
  MxState *st = (MxState *)pst;
  // partials laid out as red_partials in cg_mixed_t
  double *val = (double *)pval, *part = (double *)ppart;
  double *const R2[2] = {part + kMxR2, part + kMxR2b};
  // zero p and t so that sites no sweep writes hold finite values
  QS_CUDA(cudaMemsetAsync(P[0], 0, sizeof(uint4) * (size_t)nh, stream()));
  QS_CUDA(cudaMemsetAsync(P[1], 0, sizeof(uint4) * (size_t)nh, stream()));
  QS_CUDA(cudaMemsetAsync(t, 0, sizeof(uint4) * (size_t)nh, stream()));
  MxState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.r2req = r2req;
  hs.maxits = maxits;
  hs.delta = delta;
  {
    double *buf = host_results();
    std::memcpy(buf, &hs, sizeof(hs));
    QS_CUDA(cudaMemcpyAsync(st, buf, sizeof(hs), cudaMemcpyHostToDevice, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));
  }
  const int grid = std::min(grid_for(n, kBlock, 4), kMaxRedBlocks);
  const int egrid = grid_for(n, kBlock, 8);
  // the summed value at val[0], over processes
  auto sum_over = [&](const double *partials, int np) -> int {
    mxd_sum_kernel<<<1, kBlock, 0, stream()>>>(partials, np, val);
    note_launch();
    QS_LAUNCH_CHECK();
    return D.allreduce(D.ctx, val, 1);
  };
  mxd_init_kernel<VP><<<grid, kBlock, 0, stream()>>>(b, x, r, rs, xs, PI[0], n, part);
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = sum_over(part, grid))) return rc;
  mxd_init_state_kernel<<<1, 1, 0, stream()>>>(st, val);
  note_launch();
  DslashArgsLo A1, A2;
  A1.g = geo;
  A1.L = lo_links(g->low, PREC);
  A1.halt = st;
  A1.partials = part;
  A1.ticket = red_tickets();
  A1.dot_out = nullptr;
  A1.po = 1;
  A1.xin = P[0];
  A1.istride = nh;
  A1.xs = nullptr;
  A1.sstride = 0;
  A1.out = t;
  A1.ostride = nh;
  A1.b = 0.f;
  A1.k_lo = D.odd_lo;
  A1.k_hi = D.odd_hi;
  A2 = A1;
  A2.po = 0;
  A2.xin = t;
  A2.xs = P[0];
  A2.sstride = nh;
  A2.out = ap;
  A2.ostride = n;
  A2.out_off = D.even_lo;
  A2.b = (float)(4.0 * m2);
  A2.k_lo = D.even_lo;
  A2.k_hi = D.even_lo + n;
  A2.rdot = rs;  // Re <r, Ap> partials (interior sites, as ap)
  // The three-kernel iteration of cg_mixed_t with one sum over the
  // processes per iteration: the ghost exchange of P[cur], the half sweeps,
  // then <p, Ap>, |Ap|^2, <r, Ap> and the previous update's |r|^2 summed in
  // the domain and over the processes together, then the fused update.
  int cur = 0;
  bool fresh = true;
  auto iteration = [&]() -> int {
    int rc2 = D.exchange_even(D.ctx, P[cur]);
    if (rc2) return rc2;
    int np = 0;
    A1.xin = P[cur];
    A2.xs = P[cur];
    if ((rc2 = g->nl == 8 ? sloppy_half<PREC, 8>(0, A1, 0, 0, nullptr) : sloppy_half<PREC, 4>(0, A1, 0, 0, nullptr)))
      return rc2;
    if ((rc2 = g->nl == 8 ? sloppy_half<PREC, 8>(1, A2, 0, 4, &np) : sloppy_half<PREC, 4>(1, A2, 0, 4, &np)))
      return rc2;
    mxd_sum4_kernel<<<1, kBlock, 0, stream()>>>(part, part + kMxApAp, part + kMxRAp, np, R2[cur],
                                                fresh ? 0 : grid, val);
    note_launch();
    QS_LAUNCH_CHECK();
    if ((rc2 = D.allreduce(D.ctx, val, 4))) return rc2;
    launch_pdl(mx_update_p_kernel<VP>, grid, kBlock, rs, xs, (const float2 *)ap, (const void *)PI[cur],
               (void *)PI[cur ^ 1], n, st, (const double *)val, (const double *)(val + 1), 1,
               (const double *)(val + 2), fresh ? 0 : 1, R2[cur ^ 1], cur, (const double *)(val + 3));
    note_launch();
    QS_LAUNCH_CHECK();
    cur ^= 1;
    fresh = false;
    return QEXSTAG_OK;
  };
  // the direction corrected is the one the last update that ran read
  // (PI[hs.pin]); the iteration goes on from it
  auto reliable_update = [&](int pin) -> int {
    mx_flush_kernel<<<egrid, kBlock, 0, stream()>>>(x, xs, n);
    note_launch();
    int rc2 = D.schur64(D.ctx, x, ax);
    if (rc2) return rc2;
    cur = pin & 1;
    fresh = true;
    mxd_true_res_kernel<<<grid, kBlock, 0, stream()>>>(b, ax, r, rs, n, part);
    note_launch();
    if ((rc2 = sum_over(part, grid))) return rc2;
    mxd_true_res_state_kernel<<<1, 1, 0, stream()>>>(st, val);
    mxd_rp_kernel<VP><<<grid, kBlock, 0, stream()>>>(rs, PI[cur], n, part);
    note_launch(2);
    if ((rc2 = sum_over(part, grid))) return rc2;
    mxd_set_rp_kernel<<<1, 1, 0, stream()>>>(st, val);
    mx_p_reliable_kernel<VP><<<egrid, kBlock, 0, stream()>>>(rs, PI[cur], n, st);
    mx_clear_pending_kernel<<<1, 1, 0, stream()>>>(st);
    note_launch(3);
    QS_LAUNCH_CHECK();
    return QEXSTAG_OK;
  };
  // every process sees the same summed state, so all run the same batches
  // (kernels past convergence or a pending update return at once)
  const int every = check_interval(n);
  StateSnapshot snap;
  for (;;) {
    for (int i = 0; i < every; i++)
      if ((rc = iteration())) return rc;
    if ((rc = snap.start(st, sizeof(MxState))) || (rc = snap.wait(&hs, sizeof(MxState)))) return rc;
    if (hs.done) break;
    if (hs.pending && (rc = reliable_update(hs.pin))) return rc;
  }
  out->iterations = hs.itn;
  out->r2 = hs.b2 > 0 ? hs.r2 / hs.b2 : 0.0;
  out->nan = hs.nan;
  *reliable = hs.reliable;
  if (hs.nan) return fail(QEXSTAG_ERR_NAN, "domain mixed cg: NaN in residual");
  return QEXSTAG_OK;
}

}  // namespace qs

// ---------------------------------------------------------------------------
// timing of the Schur operator in each precision (benchmark hook)
// ---------------------------------------------------------------------------
namespace qs {

template <int PREC>
__global__ void fill_vec_kernel(void *p, int n, unsigned seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 v[3];
    unsigned h = (unsigned)i * 2654435761u + seed;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      h ^= h >> 13;
      h *= 0x5bd1e995u;
      float a = (float)(h & 0xffff) * (1.f / 65536.f) - 0.5f;
      h ^= h >> 15;
      h *= 0x27d4eb2du;
      float b = (float)(h & 0xffff) * (1.f / 65536.f) - 0.5f;
      v[c] = make_float2(a, b);
    }
    store_vec<PREC>(p, n, i, v);
  }
}

__global__ void fill_vec64_kernel(double2 *p, int n, unsigned seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) {
    unsigned h = (unsigned)i * 2654435761u + seed;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    p[i] = make_double2((double)(h & 0xffff) / 65536.0 - 0.5, (double)((h >> 16) & 0xffff) / 65536.0 - 0.5);
  }
}

int bench_schur(qexstag_links_s *g, int prec, int nrep, double m2, double *sec) {
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  Workspace &ws = g->ws;
  void *pa, *pb, *pc;
  int rc;
  const size_t v64 = sizeof(double2) * 3 * (size_t)nh;
  if ((rc = ws.get(kSlotMx0 + 20, v64, &pa)) || (rc = ws.get(kSlotMx0 + 21, v64, &pb)) ||
      (rc = ws.get(kSlotMx0 + 22, v64, &pc)))
    return rc;
  const int grid = grid_for(nh);
  if (prec == 0) {
    fill_vec64_kernel<<<grid, kBlock, 0, stream()>>>((double2 *)pa, nh, 1u);
  } else if (prec == 1) {
    fill_vec_kernel<kF32><<<grid, kBlock, 0, stream()>>>(pa, nh, 1u);
  } else {
    fill_vec_kernel<VecPrec<kF16>::v><<<grid, kBlock, 0, stream()>>>(pa, nh, 1u);
  }
  note_launch();
  QS_LAUNCH_CHECK();
  auto once = [&]() -> int {
    if (prec == 0)
      return schur64(g, 0, VecD{(double2 *)pc, nh}, CVecD{(const double2 *)pa, nh}, VecD{(double2 *)pb, nh}, m2);
    return schur_lo(g, prec == 1 ? kF32 : kF16, 0, (float2 *)pc, pa, pb, m2, 0, nullptr, nullptr, nullptr);
  };
  for (int i = 0; i < 2; i++)
    if ((rc = once())) return rc;
  cudaEvent_t e0, e1;
  QS_CUDA(cudaEventCreate(&e0));
  QS_CUDA(cudaEventCreate(&e1));
  QS_CUDA(cudaEventRecord(e0, stream()));
  for (int i = 0; i < nrep; i++)
    if ((rc = once())) break;
  cudaEventRecord(e1, stream());
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  *sec = ms * 1e-3 / nrep;
  return QEXSTAG_OK;
}

}  // namespace qs

extern "C" int qexstag_bench_schur(qexstag_links *g, int prec, int nrep, double m2,
                                   double *seconds_per_call) {
  if (!g || !g->u64 || !seconds_per_call || nrep < 1 || prec < 0 || prec > 2)
    return qs::fail(QEXSTAG_ERR_ARG, "bench_schur: bad argument");
  int rc = qs::runtime_ready();
  if (rc) return rc;
  return qs::bench_schur(g, prec, nrep, m2, seconds_per_call);
}
