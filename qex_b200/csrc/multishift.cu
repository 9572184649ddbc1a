// multishift.cu -- multi-shift CG (src/solvers/cgm.nim:68-246, after
// Jegerlehner, hep-lat/9612014) for several right-hand sides at once, and
// the drivers built on it:
//   solve_multishift: QEX's multi-mass solve (stagSolve.nim:560-668), FP64,
//     one right-hand side, every shift updated every iteration as cgm.nim does;
//   cgm_ee: (A + sigma_k) y_jk = b_j for up to 8 right-hand sides, with an
//     FP32 multi-right-hand-side Dslash that reads each link once per site for
//     all of them, shifts dropped once their residual |zeta_k| |r| meets the
//     target, then FP64 true residuals and, for every shift, a
//     multi-right-hand-side FP32 CG on the residuals of the right-hand sides
//     still above it (FP64 defect correction).
// All scalars (alpha, beta, zeta recurrences) live on the device in FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lib.cuh"
#include "lowprec.cuh"

namespace qs {

constexpr int kMaxShift = 32;
constexpr int kMaxRhs = 8;

struct CgmState {
  int itn, maxits, done, dropping;
  int nshift, nrhs, pad0, pad1;
  int live[kMaxRhs];  // right-hand side still iterating this iteration
  int cont[kMaxRhs];  // continuing after this iteration
  double r2i[kMaxRhs], pAp[kMaxRhs], alpha[kMaxRhs], beta[kMaxRhs];
  double alphaim1[kMaxRhs], betaim1[kMaxRhs], r2stop[kMaxRhs], b2[kMaxRhs];
  double sg[kMaxShift];
  double zi[kMaxRhs][kMaxShift], zim1[kMaxRhs][kMaxShift];
  double cx[kMaxRhs][kMaxShift], cr[kMaxRhs][kMaxShift], cp[kMaxRhs][kMaxShift];
  int dox[kMaxRhs][kMaxShift], dop[kMaxRhs][kMaxShift], active[kMaxRhs][kMaxShift];
};

// vectors of the solve: [nrhs][3][nh] (r, Ap, t) and [nrhs][nshift][3][nh]
// (x, p); element type double2 (FP64) or float2 (FP32)
template <class VT>
struct CgmVecs {
  VT *r, *ap, *t, *x, *p;
  int nh, nshift, nrhs;
  __host__ __device__ size_t rhs_off(int j) const { return (size_t)j * 3 * nh; }
  __host__ __device__ size_t xs_off(int j, int k) const { return ((size_t)j * nshift + k) * 3 * nh; }
};

// ---------------------------------------------------------------------------
// FP32 multi-right-hand-side Dslash: a block is kMrhsGroups warp-uniform
// groups of kMrhsSites sites; group q applies the operator to right-hand
// sides q*kMrhsPer .. q*kMrhsPer+kMrhsPer-1 of its sites.  Every group loads
// the same links, so each link comes from HBM once per site and from L1 for
// the other groups, while each right-hand side's vector loads stay
// coalesced across the warp.
// ---------------------------------------------------------------------------

constexpr int kMrhsPer = 4;                       // right-hand sides per thread
constexpr int kMrhsGroups = kMaxRhs / kMrhsPer;   // 2
constexpr int kMrhsSites = kBlock / kMrhsGroups;  // 128 sites per block step

struct MrhsArgs {
  Geom g;
  int po, nr;
  LoLinks L;
  const float2 *xin;  // [nr][3][nh]
  const float2 *xs;   // [nr][3][nh] same-site operand (INIT)
  float2 *out;        // [nr][3][nh]
  size_t irs, srs, ors;  // right-hand-side strides of xin, xs, out
  int nh;
  float b;
  const CgmState *st;
  CgmState *wst;
  double *partials;
  unsigned *ticket;
};

template <int NL, int HOP, int INIT, int RED, int R12>
__global__ void __launch_bounds__(kBlock, 2) dslash_mrhs_kernel(const MrhsArgs A) {
  pdl_wait();
  if (A.st->done) return;
  const Geom &g = A.g;
  const int nh = g.nh;
  const size_t V = (size_t)g.V;
  const size_t in_base = (size_t)(1 - A.po) * nh;
  const size_t out_base = (size_t)A.po * nh;
  const int grp = threadIdx.x / kMrhsSites;
  const int j0 = grp * kMrhsPer;
  double dot[kMrhsPer];
#pragma unroll
  for (int q = 0; q < kMrhsPer; q++) dot[q] = 0.0;
  for (int k = blockIdx.x * kMrhsSites + (threadIdx.x % kMrhsSites); k < nh; k += gridDim.x * kMrhsSites) {
    if (j0 >= A.nr) break;
    int x[4], lex;
    site_coords(g, A.po, k, x, lex);
    float2 acc[kMrhsPer][3];
#pragma unroll
    for (int q = 0; q < kMrhsPer; q++)
#pragma unroll
      for (int c = 0; c < 3; c++) acc[q][c] = make_float2(0.f, 0.f);
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const bool is_long = (NL == 8) && (l & 1);
      const int f = (NL == 8) ? (l >> 1) : l;
      const int jf = nbr_half(g, x, lex, mu, len);
      const int jb = nbr_half(g, x, lex, mu, -len);
      float2 uf[9], ub[9];
      if (is_long && R12) {
        load_long12<kF32>(A.L, f, out_base + k, V, long_sign_fwd(g, x, mu), uf);
        load_long12<kF32>(A.L, f, in_base + jb, V, long_sign_bck(g, x, mu), ub);
      } else if (is_long) {
        load_link18<kF32>(A.L.f32_long, A.L.f32_long_tail, nullptr, nullptr, f, out_base + k, V, uf);
        load_link18<kF32>(A.L.f32_long, A.L.f32_long_tail, nullptr, nullptr, f, in_base + jb, V, ub);
      } else {
        load_link18<kF32>(A.L.f32_fat, A.L.f32_fat_tail, nullptr, nullptr, f, out_base + k, V, uf);
        load_link18<kF32>(A.L.f32_fat, A.L.f32_fat_tail, nullptr, nullptr, f, in_base + jb, V, ub);
      }
#pragma unroll
      for (int q = 0; q < kMrhsPer; q++) {
        const int j = j0 + q;
        if (j < A.nr) {
          const float2 *xj = A.xin + (size_t)j * A.irs;
          float2 v[3], w[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            v[c] = ldg(xj + (size_t)c * nh + jf);
            w[c] = ldg(xj + (size_t)c * nh + jb);
          }
#pragma unroll
          for (int i = 0; i < 3; i++) {
            float2 t = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 3; c++) {
              t = cmadd(t, uf[3 * i + c], v[c]);
              u = cjmadd(u, ub[3 * c + i], w[c]);
            }
            if (HOP > 0) {
              acc[q][i].x += t.x - u.x;
              acc[q][i].y += t.y - u.y;
            } else {
              acc[q][i].x -= t.x - u.x;
              acc[q][i].y -= t.y - u.y;
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kMrhsPer; q++) {
      const int j = j0 + q;
      if (j < A.nr) {
        float2 *oj = A.out + (size_t)j * A.ors;
        float d = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          float2 o = acc[q][c];
          if (INIT) {
            float2 s = __ldcg(A.xs + (size_t)j * A.srs + (size_t)c * nh + k);
            o.x = fmaf(A.b, s.x, o.x);
            o.y = fmaf(A.b, s.y, o.y);
            if (RED) d += s.x * o.x + s.y * o.y;
          }
          oj[(size_t)c * nh + k] = o;
        }
        if (RED) dot[q] += (double)d;
      }
    }
  }
  if (RED) {
    // each right-hand side's sum from its group's threads (static indices)
    double all[kMaxRhs];
#pragma unroll
    for (int j = 0; j < kMaxRhs; j++) all[j] = (j / kMrhsPer == grp) ? dot[j % kMrhsPer] : 0.0;
    double s[kMaxRhs];
    if (grid_reduce<kMaxRhs>(all, A.partials, A.ticket, s) && threadIdx.x == 0)
      for (int j = 0; j < A.nr; j++) A.wst->pAp[j] = s[j];
  }
}

template <int NL, int R12>
static void mrhs_pair(MrhsArgs A, int par, const float2 *p, size_t prs, float2 *t, float2 *ap, float b4m2,
                      int grid) {
  const size_t vs = (size_t)3 * A.nh;
  A.po = 1 - par;
  A.xin = p;
  A.irs = prs;
  A.xs = nullptr;
  A.srs = 0;
  A.out = t;
  A.ors = vs;
  A.b = 0.f;
  launch_pdl(dslash_mrhs_kernel<NL, 1, 0, 0, R12>, grid, kBlock, A);
  A.po = par;
  A.xin = t;
  A.irs = vs;
  A.xs = p;
  A.srs = prs;
  A.out = ap;
  A.ors = vs;
  A.b = b4m2;
  launch_pdl(dslash_mrhs_kernel<NL, -1, 1, 1, R12>, grid, kBlock, A);
  note_launch(2);
}

// p_j at p + j*prs; t_j, ap_j at j*3*nh
static int schur_mrhs(const qexstag_links_s *g, int par, int nr, const float2 *p, size_t prs, float2 *t,
                      float2 *ap, double m2, CgmState *st) {
  const Geom &geo = g->l->g;
  MrhsArgs A;
  A.g = geo;
  A.nr = nr;
  A.L = lo_links(g->low, kF32);
  A.nh = geo.nh;
  A.st = st;
  A.wst = st;
  A.partials = red_partials();
  A.ticket = red_tickets();
  // blocks step over kMrhsSites sites; at most kMaxRedBlocks*8/kMaxRhs for the reduction
  int grid = (int)std::min<long>(((long)geo.nh + kMrhsSites - 1) / kMrhsSites, (long)num_sms() * 4);
  if (grid * kMaxRhs > kMaxRedBlocks * 8) grid = kMaxRedBlocks * 8 / kMaxRhs;
  if (grid < 1) grid = 1;
  const float b4 = (float)(4.0 * m2);
  if (g->nl == 8) {
    if (g->low.recon12)
      mrhs_pair<8, 1>(A, par, p, prs, t, ap, b4, grid);
    else
      mrhs_pair<8, 0>(A, par, p, prs, t, ap, b4, grid);
  } else {
    mrhs_pair<4, 0>(A, par, p, prs, t, ap, b4, grid);
  }
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// CG-M iteration kernels (element type VT)
// ---------------------------------------------------------------------------

__global__ void cgm_alpha_kernel(CgmState *st) {
  if (st->done) return;
  for (int j = 0; j < st->nrhs; j++) {
    double pAp = st->pAp[j];
    st->alpha[j] = (pAp != 0.0) ? st->r2i[j] / pAp : 0.0;
  }
  st->itn += 1;
}

template <class VT>
__device__ __forceinline__ VT vload(const VT *p) { return *p; }

__device__ __forceinline__ void axpy2(double2 &y, double a, double2 x) {
  y.x = fma(a, x.x, y.x);
  y.y = fma(a, x.y, y.y);
}
__device__ __forceinline__ void axpy2(float2 &y, double a, float2 x) {
  y.x = fmaf((float)a, x.x, y.x);
  y.y = fmaf((float)a, x.y, y.y);
}

// cgm.nim:157-184 for shift 0: r -= alpha Ap; x0 += alpha p0; |r|^2; then the
// zeta recurrences of every other shift (cgm.nim:187-200)
template <class VT>
__global__ void __launch_bounds__(kBlock) cgm_update1_kernel(CgmVecs<VT> v, CgmState *st, double *partials,
                                                            unsigned *ticket) {
  if (st->done) return;
  const int nh = v.nh;
  double s[kMaxRhs];
#pragma unroll
  for (int j = 0; j < kMaxRhs; j++) s[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < kMaxRhs; j++) {
      if (j < v.nrhs && st->live[j]) {
        const double a = st->alpha[j];
        VT *r = v.r + v.rhs_off(j);
        const VT *ap = v.ap + v.rhs_off(j);
        VT *x0 = v.x + v.xs_off(j, 0);
        const VT *p0 = v.p + v.xs_off(j, 0);
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const size_t o = (size_t)c * nh + i;
          VT rv = r[o], xv = x0[o];
          axpy2(rv, -a, ap[o]);
          axpy2(xv, a, p0[o]);
          r[o] = rv;
          x0[o] = xv;
          acc += (double)rv.x * rv.x + (double)rv.y * rv.y;
        }
        s[j] += acc;
      }
    }
  }
  double tot[kMaxRhs];
  if (!(grid_reduce<kMaxRhs>(s, partials, ticket, tot) && threadIdx.x == 0)) return;
  for (int j = 0; j < st->nrhs; j++) {
    if (!st->live[j]) continue;
    const double alpha = st->alpha[j], r2i = st->r2i[j];
    const double r2ip1 = tot[j];
    const double beta = (r2i != 0.0) ? r2ip1 / r2i : 0.0;
    const bool cont = (st->itn < st->maxits) && (r2ip1 > st->r2stop[j]);
    st->beta[j] = beta;
    for (int k = 1; k < st->nshift; k++) {
      if (!st->active[j][k]) {
        st->dox[j][k] = st->dop[j][k] = 0;
        continue;
      }
      const double zi = st->zi[j][k], zim1 = st->zim1[j][k], sg = st->sg[k];
      double zip1d = alpha * st->betaim1[j] * (zim1 - zi);
      zip1d += zim1 * st->alphaim1[j] * (1.0 + sg * alpha);
      const double zip1 = (zip1d != 0.0) ? zi * zim1 * st->alphaim1[j] / zip1d : 0.0;
      const double zr = (zi != 0.0) ? zip1 / zi : 0.0;
      st->cx[j][k] = alpha * zr;
      st->dox[j][k] = 1;
      st->dop[j][k] = cont ? 1 : 0;
      if (cont) {
        st->cr[j][k] = zip1;
        st->cp[j][k] = beta * zr * zr;
        st->zim1[j][k] = zi;
        st->zi[j][k] = zip1;
        // the shifted residual is zeta_k r: stop updating a shift that meets it
        if (st->dropping && zip1 * zip1 * r2ip1 <= st->r2stop[j]) st->active[j][k] = 0;
      }
    }
    st->alphaim1[j] = alpha;
    st->betaim1[j] = beta;
    st->r2i[j] = r2ip1;
    st->cont[j] = cont ? 1 : 0;
  }
}

// p0 = r + beta p0; x_k += cx p_k; p_k = cr r + cp p_k
template <class VT>
__global__ void cgm_update2_kernel(CgmVecs<VT> v, const CgmState *st) {
  if (st->done) return;
  const int nh = v.nh;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
    for (int j = 0; j < v.nrhs; j++) {
      if (!st->live[j]) continue;
      const VT *r = v.r + v.rhs_off(j);
      VT rv[3];
#pragma unroll
      for (int c = 0; c < 3; c++) rv[c] = r[(size_t)c * nh + i];
      if (st->cont[j]) {
        VT *p0 = v.p + v.xs_off(j, 0);
        const double b = st->beta[j];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const size_t o = (size_t)c * nh + i;
          VT pv = p0[o];
          VT q = rv[c];
          axpy2(q, b, pv);
          p0[o] = q;
        }
      }
      for (int k = 1; k < v.nshift; k++) {
        if (!st->dox[j][k]) continue;
        VT *xk = v.x + v.xs_off(j, k);
        VT *pk = v.p + v.xs_off(j, k);
        const double cx = st->cx[j][k];
        const bool dp = st->dop[j][k];
        const double cr = st->cr[j][k], cp = st->cp[j][k];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const size_t o = (size_t)c * nh + i;
          VT pv = pk[o], xv = xk[o];
          axpy2(xv, cx, pv);
          xk[o] = xv;
          if (dp) {
            VT q;
            q.x = 0;
            q.y = 0;
            axpy2(q, cr, rv[c]);
            axpy2(q, cp, pv);
            pk[o] = q;
          }
        }
      }
    }
  }
}

__global__ void cgm_finish_kernel(CgmState *st) {
  if (st->done) return;
  int any = 0;
  for (int j = 0; j < st->nrhs; j++) {
    st->live[j] = st->cont[j];
    any |= st->cont[j];
  }
  if (!any) st->done = 1;
}

// initial state: r = b, x = 0, p_k = r; |b|^2 per right-hand side
template <class VT>
__global__ void __launch_bounds__(kBlock) cgm_init_kernel(CgmVecs<VT> v, const double2 *const *b, int bstride,
                                                         CgmState *st, double *partials, unsigned *ticket,
                                                         double r2req) {
  const int nh = v.nh;
  double s[kMaxRhs];
#pragma unroll
  for (int j = 0; j < kMaxRhs; j++) s[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < kMaxRhs; j++) {
      if (j < v.nrhs) {
        const double2 *bj = b[j];
        double acc = 0.0;
        for (int c = 0; c < 3; c++) {
          double2 bv = bj[(size_t)c * bstride + i];
          VT rv;
          rv.x = bv.x;
          rv.y = bv.y;
          v.r[v.rhs_off(j) + (size_t)c * nh + i] = rv;
          VT z;
          z.x = 0;
          z.y = 0;
          for (int k = 0; k < v.nshift; k++) {
            v.x[v.xs_off(j, k) + (size_t)c * nh + i] = z;
            v.p[v.xs_off(j, k) + (size_t)c * nh + i] = rv;
          }
          acc += bv.x * bv.x + bv.y * bv.y;
        }
        s[j] += acc;
      }
    }
  }
  double tot[kMaxRhs];
  if (!(grid_reduce<kMaxRhs>(s, partials, ticket, tot) && threadIdx.x == 0)) return;
  int any = 0;
  st->itn = 0;
  for (int j = 0; j < st->nrhs; j++) {
    st->b2[j] = tot[j];
    st->r2i[j] = tot[j];
    st->r2stop[j] = r2req * tot[j];
    st->alphaim1[j] = -1.0;
    st->betaim1[j] = 0.0;
    const int c = (tot[j] > st->r2stop[j]) && isfinite(tot[j]) ? 1 : 0;
    st->cont[j] = st->live[j] = c;
    any |= c;
    for (int k = 0; k < st->nshift; k++) {
      st->zi[j][k] = st->zim1[j][k] = 1.0;
      st->active[j][k] = 1;
      st->dox[j][k] = st->dop[j][k] = 0;
    }
  }
  st->done = (any && st->maxits > 0) ? 0 : 1;
}

// FP32 or FP64 vector -> FP64 block of a full-lattice field
template <class VT>
__global__ void cgm_out_kernel(const VT *x, int nh, double2 *y, int ystride, double scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x)
    for (int c = 0; c < 3; c++) {
      VT v = x[(size_t)c * nh + i];
      y[(size_t)c * ystride + i] = make_double2(scale * (double)v.x, scale * (double)v.y);
    }
}

static int read_cgm_head(const CgmState *d, CgmState *h) {
  double *buf = host_results();
  const size_t n = offsetof(CgmState, r2i);
  QS_CUDA(cudaMemcpyAsync(buf, d, n, cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  std::memcpy(h, buf, n);
  return QEXSTAG_OK;
}

int check_interval(int nh);
int schur_lo_v32(const qexstag_links_s *g, int prec, int par, float2 *ap, const float2 *p, float2 *t, double m2,
                 double *dot_out);
int cg_mixed(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits, int sloppy,
             double delta, CgOut *out, int *reliable);

// Multi-shift CG on parity par: (A + sg[k]) x_jk = b_j, A = stagD2xx(m2),
// sg[0] = 0.  fp32: FP32 vectors with the multi-rhs FP32 Dslash (one
// right-hand side: the single-vector sloppy Schur with links of precision
// lprec, kF32 or kF16), else FP64 (nrhs must be 1).  Solutions are written
// to y[j*nshift+k] (FP64 blocks of parity par with stride ystride) scaled by
// yscale.
static int cgm_core(qexstag_links_s *g, int par, double m2, int nshift, const double *sg, int nrhs,
                    const double2 *const *b, int bstride, double2 *const *y, int ystride, double yscale,
                    double r2req, int maxits, bool fp32, bool dropping, int *iters, int lprec = kF32) {
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  Workspace &ws = g->ws;
  const size_t es = fp32 ? sizeof(float2) : sizeof(double2);
  const size_t vb = es * 3 * (size_t)nh;
  void *pr, *pap, *pt, *px, *pp, *pst, *pb;
  int rc;
  if ((rc = ws.get(kSlotMs0 + 40, vb * nrhs, &pr)) || (rc = ws.get(kSlotMs0 + 41, vb * nrhs, &pap)) ||
      (rc = ws.get(kSlotMs0 + 42, vb * nrhs, &pt)) || (rc = ws.get(kSlotMs0 + 43, vb * nrhs * nshift, &px)) ||
      (rc = ws.get(kSlotMs0 + 44, vb * nrhs * nshift, &pp)) ||
      (rc = ws.get(kSlotMs0 + 45, sizeof(CgmState), &pst)) ||
      (rc = ws.get(kSlotMs0 + 46, sizeof(double2 *) * kMaxRhs, &pb)))
    return rc;
  CgmState *st = (CgmState *)pst;
  CgmState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.maxits = maxits;
  hs.nshift = nshift;
  hs.nrhs = nrhs;
  hs.dropping = dropping ? 1 : 0;
  for (int k = 0; k < nshift; k++) hs.sg[k] = (k == 0) ? 0.0 : sg[k];
  std::vector<char> staging(sizeof(CgmState) + sizeof(double2 *) * kMaxRhs);
  void *pin;
  if ((rc = ws.get_pinned(staging.size(), &pin))) return rc;
  std::memcpy(pin, &hs, sizeof(hs));
  std::memcpy((char *)pin + sizeof(hs), b, sizeof(double2 *) * nrhs);
  QS_CUDA(cudaMemcpyAsync(st, pin, sizeof(hs), cudaMemcpyHostToDevice, stream()));
  QS_CUDA(cudaMemcpyAsync(pb, (char *)pin + sizeof(hs), sizeof(double2 *) * nrhs, cudaMemcpyHostToDevice,
                          stream()));
  const int grid = std::min(grid_for(nh, kBlock, 4), kMaxRedBlocks * 8 / kMaxRhs);
  const int egrid = grid_for(nh, kBlock, 8);
  const int every = check_interval(nh);
  if (fp32) {
    CgmVecs<float2> v{(float2 *)pr, (float2 *)pap, (float2 *)pt, (float2 *)px, (float2 *)pp, nh, nshift, nrhs};
    cgm_init_kernel<float2><<<grid, kBlock, 0, stream()>>>(v, (const double2 *const *)pb, bstride, st,
                                                           red_partials(), red_tickets(), r2req);
    note_launch();
    QS_LAUNCH_CHECK();
    for (;;) {
      for (int i = 0; i < every; i++) {
        // p_0 of right-hand side j lives at xs_off(j, 0)
        if (nrhs == 1)
          rc = schur_lo_v32(g, lprec, par, v.ap, v.p, v.t, m2, &st->pAp[0]);
        else
          rc = schur_mrhs(g, par, nrhs, v.p, v.xs_off(1, 0), v.t, v.ap, m2, st);
        if (rc) return rc;
        cgm_alpha_kernel<<<1, 1, 0, stream()>>>(st);
        cgm_update1_kernel<float2><<<grid, kBlock, 0, stream()>>>(v, st, red_partials(), red_tickets());
        cgm_update2_kernel<float2><<<egrid, kBlock, 0, stream()>>>(v, st);
        cgm_finish_kernel<<<1, 1, 0, stream()>>>(st);
        note_launch(4);
      }
      QS_LAUNCH_CHECK();
      if ((rc = read_cgm_head(st, &hs))) return rc;
      if (hs.done) break;
    }
    for (int j = 0; j < nrhs; j++)
      for (int k = 0; k < nshift; k++) {
        cgm_out_kernel<float2><<<egrid, kBlock, 0, stream()>>>(v.x + v.xs_off(j, k), nh, y[j * nshift + k],
                                                               ystride, yscale);
        note_launch();
      }
  } else {
    if (nrhs != 1) return fail(QEXSTAG_ERR_ARG, "FP64 multi-shift takes one right-hand side");
    CgmVecs<double2> v{(double2 *)pr, (double2 *)pap, (double2 *)pt, (double2 *)px, (double2 *)pp, nh, nshift, 1};
    cgm_init_kernel<double2><<<grid, kBlock, 0, stream()>>>(v, (const double2 *const *)pb, bstride, st,
                                                            red_partials(), red_tickets(), r2req);
    note_launch();
    QS_LAUNCH_CHECK();
    for (;;) {
      for (int i = 0; i < every; i++) {
        if ((rc = schur64(g, par, VecD{v.ap, nh}, CVecD{v.p, nh}, VecD{v.t, nh}, m2, kRedDot, nullptr,
                          &st->done, &st->pAp[0])))
          return rc;
        cgm_alpha_kernel<<<1, 1, 0, stream()>>>(st);
        cgm_update1_kernel<double2><<<grid, kBlock, 0, stream()>>>(v, st, red_partials(), red_tickets());
        cgm_update2_kernel<double2><<<egrid, kBlock, 0, stream()>>>(v, st);
        cgm_finish_kernel<<<1, 1, 0, stream()>>>(st);
        note_launch(4);
      }
      QS_LAUNCH_CHECK();
      if ((rc = read_cgm_head(st, &hs))) return rc;
      if (hs.done) break;
    }
    for (int k = 0; k < nshift; k++) {
      cgm_out_kernel<double2><<<egrid, kBlock, 0, stream()>>>(v.x + v.xs_off(0, k), nh, y[k], ystride, yscale);
      note_launch();
    }
  }
  QS_LAUNCH_CHECK();
  *iters = hs.itn;
  return QEXSTAG_OK;
}

int apply_D(qexstag_links_s *g, double2 *r, const double2 *x, double m, double sc);

// QEX's multi-mass solve (stagSolve.nim:560-668)
int solve_multishift(qexstag_links_s *g, int nmass, double2 *const *xs, const double2 *b,
                     const double *ms, const qexstag_solver_params *p, qexstag_solver_stats *st) {
  if (nmass > kMaxShift) return fail(QEXSTAG_ERR_ARG, "solve_multishift: at most 32 masses");
  const Geom &geo = g->l->g;
  const int V = geo.V, nh = geo.nh;
  Workspace &ws = g->ws;
  void *pr, *pxt;
  const size_t fb = sizeof(double2) * 3 * (size_t)V;
  int rc;
  if ((rc = ws.get(kSlotFull0, fb, &pr)) || (rc = ws.get(kSlotFull1, fb, &pxt))) return rc;
  double2 *r = (double2 *)pr, *xt = (double2 *)pxt;
  const double mass = ms[0];
  double b2e = 0, b2o = 0;
  if ((rc = vnorm2(block(b, geo, 0), nh, &b2e)) || (rc = vnorm2(block(b, geo, 1), nh, &b2o))) return rc;
  const double b2 = b2e + b2o;
  if (!std::isfinite(b2)) return fail(QEXSTAG_ERR_NAN, "solve_multishift: source is not finite");
  double r2 = b2;
  const double r2stop = p->r2req * b2;
  std::vector<double> shifts(nmass);
  for (int k = 0; k < nmass; k++) shifts[k] = (k == 0) ? 0.0 : 4.0 * (ms[k] * ms[k] - mass * mass);
  if ((rc = vcopy(VecD{r, V}, CVecD{b, V}, V)) || (rc = vzero(VecD{xt, V}, V))) return rc;
  for (int k = 0; k < nmass; k++)
    if ((rc = vzero(VecD{xs[k], V}, V))) return rc;
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  while (r2 > r2stop) {
    int mx = maxits - st->iterations;
    if (mx <= 0) break;
    double req = r2stop, r2s2 = 0.5 * req;
    double rse = (b2o <= r2s2) ? req - b2o : r2s2;
    double rso = (b2e <= r2s2) ? req - b2e : r2s2;
    int par;
    if (b2e > rse) {
      req = rse / b2e;
      par = 0;
    } else if (b2o > rso) {
      req = rso / b2o;
      par = 1;
    } else {
      break;
    }
    // cgm on parity par with r as the source; x_k[par] += 4 y_k
    std::vector<double2 *> ys(nmass);
    for (int k = 0; k < nmass; k++) {
      void *q;
      if ((rc = ws.get(kSlotMs0 + 60 + k, sizeof(double2) * 3 * (size_t)nh, &q))) return rc;
      ys[k] = (double2 *)q;
    }
    const double2 *rb = r + (size_t)par * nh;
    int its = 0;
    if ((rc = cgm_core(g, par, mass * mass, nmass, shifts.data(), 1, &rb, V, ys.data(), nh, 1.0, req, mx, false,
                       false, &its)))
      return rc;
    st->iterations += its;
    st->outer_iterations += 1;
    for (int k = 0; k < nmass; k++)
      if ((rc = vaxpy(block(xs[k], geo, par), 4.0, CVecD{ys[k], nh}, nh))) return rc;
    if ((rc = apply_D(g, xt, xs[0], mass, -1.0)) || (rc = apply_D(g, r, xt, mass, 1.0))) return rc;
    if ((rc = vsub(VecD{r, V}, CVecD{b, V}, CVecD{r, V}, V))) return rc;
    if ((rc = vnorm2(block((const double2 *)r, geo, 0), nh, &b2e)) ||
        (rc = vnorm2(block((const double2 *)r, geo, 1), nh, &b2o)))
      return rc;
    r2 = b2e + b2o;
    if (std::isnan(r2)) return fail(QEXSTAG_ERR_NAN, "solve_multishift: NaN residual");
  }
  // xs[k] = Ddag(ms[k]) xs[k]; for k = 0 that is xt from the last pass
  for (int k = 0; k < nmass; k++) {
    if (k != 0 && (rc = apply_D(g, xt, xs[k], ms[k], -1.0))) return rc;
    if ((rc = vcopy(VecD{xs[k], V}, CVecD{xt, V}, V))) return rc;
  }
  st->r2 = b2 > 0 ? r2 / b2 : 0.0;
  return (r2 > r2stop) ? QEXSTAG_NOT_CONVERGED : QEXSTAG_OK;
}

int cg64(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits, CgOut *out);

// (A + sigma) y on even sites, FP64: r = b - (A + sigma) y, returns |r|^2
static int shifted_residual(qexstag_links_s *g, double m2s, const double2 *bfull, const double2 *y, double2 *r,
                            double2 *t, double *r2) {
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  int rc;
  if ((rc = schur64(g, 0, VecD{r, nh}, block(y, geo, 0), VecD{t, nh}, m2s))) return rc;
  if ((rc = vsub(VecD{r, nh}, block(bfull, geo, 0), CVecD{r, nh}, nh))) return rc;
  return vnorm2(CVecD{r, nh}, nh, r2);
}

int cgm_ee(qexstag_links_s *g, double m, int nshift, const double *sigma, int nrhs, const double2 *const *b,
           double2 *const *y, const qexstag_solver_params *p, qexstag_solver_stats *st, double *r2_out) {
  const Geom &geo = g->l->g;
  const int V = geo.V, nh = geo.nh;
  if (nshift > kMaxShift) return fail(QEXSTAG_ERR_ARG, "cgm_ee: at most 32 shifts");
  // base system: the smallest shift; the others relative to it
  int k0 = 0;
  for (int k = 1; k < nshift; k++)
    if (sigma[k] < sigma[k0]) k0 = k;
  std::vector<int> order(nshift);
  order[0] = k0;
  for (int k = 0, n = 1; k < nshift; k++)
    if (k != k0) order[n++] = k;
  std::vector<double> sg(nshift);
  for (int k = 0; k < nshift; k++) sg[k] = sigma[order[k]] - sigma[k0];
  const double m2 = m * m + 0.25 * sigma[k0];
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  const bool sloppy = p->sloppy != QEXSTAG_SLOPPY_NONE;
  int rc;
  // zero the odd halves of the outputs
  for (int i = 0; i < nrhs * nshift; i++)
    if ((rc = vzero(block(y[i], geo, 1), nh))) return rc;
  // multi-shift phase, in batches of up to 8 right-hand sides
  const double r2ms = sloppy ? std::max(p->r2req, 1e-12) : p->r2req;
  for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
    const int nr = std::min(kMaxRhs, nrhs - j0);
    const double2 *bb[kMaxRhs];
    double2 *yy[kMaxRhs * kMaxShift];
    for (int j = 0; j < nr; j++) {
      bb[j] = b[j0 + j];
      for (int k = 0; k < nshift; k++) yy[j * nshift + k] = y[(j0 + j) * nshift + order[k]];
    }
    int its = 0;
    if (sloppy) {
      // FP32 links for the multi-shift phase at either sloppy precision: the
      // shifted solutions come out as accurate as the links they were
      // iterated with (about 1e-7 relative with FP32 links, 1e-4 with 16-bit
      // ones), and the per-shift refinement below, in the call's precision,
      // then covers three decades instead of six
      rc = cgm_core(g, 0, m2, nshift, sg.data(), nr, bb, V, yy, V, 1.0, r2ms, maxits, true, true, &its, kF32);
    } else {
      rc = 0;
      for (int j = 0; j < nr && !rc; j++) {
        int it1 = 0;
        rc = cgm_core(g, 0, m2, nshift, sg.data(), 1, &bb[j], V, &yy[j * nshift], V, 1.0, r2ms, maxits, false,
                      true, &it1);
        its += it1;
      }
    }
    if (rc) return rc;
    st->iterations += its;
  }
  st->outer_iterations += 1;
  // FP64 true residuals; refine every (j, k) above the target
  const size_t vb = sizeof(double2) * 3 * (size_t)nh;
  std::vector<double> b2(nrhs);
  for (int j = 0; j < nrhs; j++) {
    if ((rc = vnorm2(block(b[j], geo, 0), nh, &b2[j]))) return rc;
    if (!std::isfinite(b2[j])) return fail(QEXSTAG_ERR_NAN, "cgm_ee: source is not finite");
  }
  int status = QEXSTAG_OK;
  double worst = 0.0;
  if (sloppy) {
    // the right-hand sides of one shift together: a multi-right-hand-side
    // FP32 CG (cgm_core with the one shift) on their FP64 residuals, y += d,
    // repeated while any is above its target
    std::vector<double2 *> rbuf(kMaxRhs), dbuf(kMaxRhs);
    void *pt;
    for (int j = 0; j < kMaxRhs; j++) {
      void *a, *c;
      if ((rc = g->ws.get(kSlotMs0 + 100 + j, vb, &a)) || (rc = g->ws.get(kSlotMs0 + 110 + j, vb, &c))) return rc;
      rbuf[j] = (double2 *)a;
      dbuf[j] = (double2 *)c;
    }
    if ((rc = g->ws.get(kSlotMs0 + 51, vb, &pt))) return rc;
    double2 *t = (double2 *)pt;
    const double zero = 0.0;
    for (int k = 0; k < nshift; k++) {
      const double m2s = m * m + 0.25 * sigma[k];
      for (int j0 = 0; j0 < nrhs; j0 += kMaxRhs) {
        const int nr = std::min(kMaxRhs, nrhs - j0);
        std::vector<double> r2(nr);
        for (int j = 0; j < nr; j++)
          if ((rc = shifted_residual(g, m2s, b[j0 + j], y[(j0 + j) * nshift + k], rbuf[j], t, &r2[j]))) return rc;
        for (int pass = 0; pass < 10 && st->iterations < maxits; pass++) {
          // systems still above target, packed to the front
          std::vector<int> live;
          double req = 1.0;
          for (int j = 0; j < nr; j++) {
            const double stop = p->r2req * b2[j0 + j];
            if (r2[j] > stop) {
              live.push_back(j);
              req = std::min(req, 0.5 * stop / r2[j]);
            }
          }
          if (live.empty()) break;
          req = std::max(req, 1e-12);  // what an FP32 inner solve can reach
          const double2 *rb[kMaxRhs];
          double2 *dy[kMaxRhs];
          for (size_t q = 0; q < live.size(); q++) {
            rb[q] = rbuf[live[q]];
            dy[q] = dbuf[live[q]];
          }
          int its = 0;
          if (live.size() == 1) {
            // one system: the reliable-update CG in the call's sloppy precision
            CgOut o{};
            int rel = 0;
            const double delta = p->delta > 0 ? p->delta : 0.1;
            if ((rc = cg_mixed(g, 0, m2s, CVecD{rb[0], nh}, VecD{dy[0], nh}, req, maxits - st->iterations,
                               p->sloppy, delta, &o, &rel)))
              return rc;
            its = o.iterations;
            st->reliable_updates += rel;
          } else if ((rc = cgm_core(g, 0, m2s, 1, &zero, (int)live.size(), rb, nh, dy, nh, 1.0, req,
                                    maxits - st->iterations, true, false, &its))) {
            return rc;
          }
          st->iterations += its;
          st->outer_iterations += 1;
          for (size_t q = 0; q < live.size(); q++) {
            const int j = live[q];
            double2 *yk = y[(j0 + j) * nshift + k];
            if ((rc = vaxpy(block(yk, geo, 0), 1.0, CVecD{dbuf[j], nh}, nh)) ||
                (rc = shifted_residual(g, m2s, b[j0 + j], yk, rbuf[j], t, &r2[j])))
              return rc;
          }
        }
        for (int j = 0; j < nr; j++) {
          const double rel2 = b2[j0 + j] > 0 ? r2[j] / b2[j0 + j] : 0.0;
          if (r2_out) r2_out[(j0 + j) * nshift + k] = rel2;
          worst = std::max(worst, rel2);
          if (r2[j] > p->r2req * b2[j0 + j]) status = QEXSTAG_NOT_CONVERGED;
        }
      }
    }
  } else {
    void *pr, *pt, *pd;
    if ((rc = g->ws.get(kSlotMs0 + 50, vb, &pr)) || (rc = g->ws.get(kSlotMs0 + 51, vb, &pt)) ||
        (rc = g->ws.get(kSlotMs0 + 52, vb, &pd)))
      return rc;
    double2 *r = (double2 *)pr, *t = (double2 *)pt, *d = (double2 *)pd;
    for (int j = 0; j < nrhs; j++) {
      for (int k = 0; k < nshift; k++) {
        const double m2s = m * m + 0.25 * sigma[k];
        double2 *yk = y[j * nshift + k];
        double r2 = 0;
        if ((rc = shifted_residual(g, m2s, b[j], yk, r, t, &r2))) return rc;
        const double r2stop = p->r2req * b2[j];
        int pass = 0;
        while (r2 > r2stop && pass < 10 && st->iterations < maxits) {
          CgOut o{};
          const int mx = maxits - st->iterations;
          if ((rc = cg64(g, 0, m2s, CVecD{r, nh}, VecD{d, nh}, 0.5 * r2stop / r2, mx, &o))) return rc;
          st->iterations += o.iterations;
          st->outer_iterations += 1;
          if ((rc = vaxpy(block(yk, geo, 0), 1.0, CVecD{d, nh}, nh))) return rc;
          if ((rc = shifted_residual(g, m2s, b[j], yk, r, t, &r2))) return rc;
          pass++;
        }
        const double rel2 = b2[j] > 0 ? r2 / b2[j] : 0.0;
        if (r2_out) r2_out[j * nshift + k] = rel2;
        worst = std::max(worst, rel2);
        if (r2 > r2stop) status = QEXSTAG_NOT_CONVERGED;
      }
    }
  }
  st->r2 = worst;
  return status;
}

}  // namespace qs
