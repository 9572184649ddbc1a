// dslash.cu -- FP64 even-odd staggered Dslash (naive and fat+Naik) and the
// Schur operator built from two half sweeps.
//
// One thread per output site.  For each hop k the thread gathers the input
// colour vector at s+d_k and s-d_k (other parity; neighbours of consecutive
// sites are nearly consecutive, so these gathers coalesce and the other-parity
// vector is served from L2 after its first read), streams the 9 complex
// elements of U_k(s) and of U_k(s-d_k) as 16-byte words, and accumulates
// U_k(s) x(s+d_k) - U_k(s-d_k)^dagger x(s-d_k) in registers (QEX stagD2,
// src/physics/stagD.nim:383-448: per k forward then backward, after the
// a*r + b*x init).  Neighbour indices come from the site coordinates
// (src/layout/qlayout.nim:108-136) rather than from tables, which saves
// 4 bytes per hop per site of HBM traffic.
//
// Compulsory HBM bytes per output site: 8 (naive) or 16 (fat+Naik) links of
// 144 B, plus 48 B in, 48 B out, plus 48 B per same-site init operand.
#include <cstring>

#include "lib.cuh"

namespace qs {

struct DslashArgs64 {
  Geom g;
  int po;
  const double2 *__restrict__ u;
  const double2 *__restrict__ xin;
  int istride;
  const double2 *xs;  // may alias out (same site, read before the write)
  int sstride;
  const double2 *rin;  // may alias out
  int rstride;
  double2 *out;
  int ostride;
  double a, b, c;
  const int *done;
  CgState *state;
  double *partials;
  unsigned *ticket;
  double *dot_out;
  // output sites: [k0, k0 + n1) then [k2, k2 + nsites - n1) of the parity
  // block (the whole block: k0 = k2 = 0, n1 = nsites = nh); with rowlen > 0
  // instead nsites / rowlen runs of rowlen sites, pitch apart, from k0
  int k0, n1, k2, nsites;
  int rowlen, pitch;
};

template <int NL, int HOP, int INIT, int RED>
__global__ void __launch_bounds__(kBlock) dslash64_kernel(const DslashArgs64 A) {
  pdl_wait();
  if (A.done != nullptr && *A.done) return;
  const Geom &g = A.g;
  const int nh = g.nh;
  const size_t V = (size_t)g.V;
  const size_t in_base = (size_t)(1 - A.po) * nh;
  const size_t out_base = (size_t)A.po * nh;
  double dot = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < A.nsites; j += gridDim.x * blockDim.x) {
    int k;
    if (A.rowlen > 0) {
      const int q = j / A.rowlen;
      k = A.k0 + q * A.pitch + (j - q * A.rowlen);
    } else {
      k = j < A.n1 ? A.k0 + j : A.k2 + (j - A.n1);
    }
    int x[4], lex;
    site_coords(g, A.po, k, x, lex);
    double2 acc[3];
    double2 xsv[3];
    if (INIT == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] = make_double2(0.0, 0.0);
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        xsv[c] = __ldcg(A.xs + (size_t)c * A.sstride + k);
        acc[c] = make_double2(A.b * xsv[c].x, A.b * xsv[c].y);
      }
      if (INIT == 2) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          double2 rv = __ldcg(A.rin + (size_t)c * A.rstride + k);
          acc[c].x = fma(A.a, rv.x, acc[c].x);
          acc[c].y = fma(A.a, rv.y, acc[c].y);
        }
      }
    }
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const int jf = nbr_half(g, x, lex, mu, len);
      const int jb = nbr_half(g, x, lex, mu, -len);
      const double2 *ul = A.u + (size_t)l * 9 * V;
      double2 v[3], w[3], uf[9], ub[9];
#pragma unroll
      for (int c = 0; c < 3; c++) v[c] = ldg(A.xin + (size_t)c * A.istride + jf);
#pragma unroll
      for (int e = 0; e < 9; e++) uf[e] = ldlink(ul + (size_t)e * V + out_base + k);
#pragma unroll
      for (int c = 0; c < 3; c++) w[c] = ldg(A.xin + (size_t)c * A.istride + jb);
#pragma unroll
      for (int e = 0; e < 9; e++) ub[e] = ldlink(ul + (size_t)e * V + in_base + jb);
      double2 t[3], q[3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        t[i] = make_double2(0.0, 0.0);
        q[i] = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          t[i] = cmadd(t[i], uf[3 * i + j], v[j]);
          q[i] = cjmadd(q[i], ub[3 * j + i], w[j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 3; i++) {
        if (HOP > 0) {
          acc[i].x += t[i].x;
          acc[i].y += t[i].y;
          acc[i].x -= q[i].x;
          acc[i].y -= q[i].y;
        } else {
          acc[i].x -= t[i].x;
          acc[i].y -= t[i].y;
          acc[i].x += q[i].x;
          acc[i].y += q[i].y;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 o = make_double2(A.c * acc[c].x, A.c * acc[c].y);
      A.out[(size_t)c * A.ostride + k] = o;
      if (RED != kRedNone) {
        // Re <xs, out>, xs is the same-site operand (p in CG's A p)
        dot = fma(xsv[c].x, o.x, dot);
        dot = fma(xsv[c].y, o.y, dot);
      }
    }
  }
  if (RED != kRedNone) {
    double v[1] = {dot}, s[1];
    if (grid_reduce<1>(v, A.partials, A.ticket, s) && threadIdx.x == 0) {
      if (RED == kRedCgPAp) {
        // cg.nim:213-215: qLAp = <q, LAp>, alpha = rz/qLAp; itn counted at Ap
        CgState *st = A.state;
        st->pAp = s[0];
        st->alpha = st->rz / s[0];
        st->itn += 1;
      } else {
        *A.dot_out = s[0];
      }
    }
  }
  (void)out_base;
}

template <int NL, int HOP, int INIT, int RED>
static void launch64(const DslashArgs64 &A, int grid) {
  launch_pdl(dslash64_kernel<NL, HOP, INIT, RED>, grid, kBlock, A);
  note_launch();
}

template <int NL>
static int dispatch64(const DslashArgs64 &A, int hop, int init, int red, int grid) {
#define QS_D64(H, I, R)                                            \
  if (hop == H && init == I && red == R) {                         \
    launch64<NL, H, I, R>(A, grid);                                \
    return QEXSTAG_OK;                                             \
  }
  QS_D64(1, 0, kRedNone)
  QS_D64(1, 1, kRedNone)
  QS_D64(1, 2, kRedNone)
  QS_D64(-1, 0, kRedNone)
  QS_D64(-1, 1, kRedNone)
  QS_D64(-1, 2, kRedNone)
  QS_D64(-1, 1, kRedCgPAp)
  QS_D64(-1, 1, kRedDot)
#undef QS_D64
  return fail(QEXSTAG_ERR_ARG, "dslash64: unsupported variant");
}

int dslash64(const qexstag_links_s *gl, int po, VecD out, CVecD xin, CVecD xs, CVecD rin,
             double a, double b, double c, int hop, int init, int red, void *state,
             const int *done, double *dot_out) {
  const Geom &g = gl->l->g;
  DslashArgs64 A;
  A.g = g;
  A.po = po;
  A.u = gl->u64;
  A.xin = xin.p;
  A.istride = xin.stride;
  A.xs = xs.p;
  A.sstride = xs.stride;
  A.rin = rin.p;
  A.rstride = rin.stride;
  A.out = out.p;
  A.ostride = out.stride;
  A.a = a;
  A.b = b;
  A.c = c;
  A.done = done;
  A.state = (CgState *)state;
  A.partials = red_partials();
  A.ticket = red_tickets();
  A.dot_out = dot_out;
  A.k0 = A.k2 = 0;
  A.n1 = A.nsites = g.nh;
  A.rowlen = A.pitch = 0;
  int grid = grid_for(g.nh, kBlock, 6);
  if (red != kRedNone && grid > kMaxRedBlocks) grid = kMaxRedBlocks;
  int rc = (gl->nl == 8) ? dispatch64<8>(A, hop, init, red, grid)
                         : dispatch64<4>(A, hop, init, red, grid);
  if (rc) return rc;
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// One half sweep over the sites [k0, k1) and [k2, k3) of parity po (either
// range may be empty): out = b xs + c (2D) xin with hop sign hop, no
// reduction; skipped once *done is set.  Used for the halo-overlapped
// Schur operator of a domain, whose interior sweeps run while the ghost
// slices are in flight.
int dslash64_ranges(const qexstag_links_s *gl, int po, VecD out, CVecD xin, CVecD xs, double b, double c,
                    int hop, int k0, int k1, int k2, int k3, const int *done) {
  const Geom &g = gl->l->g;
  if (k0 < 0 || k1 < k0 || k2 < 0 || k3 < k2 || k1 > g.nh || k3 > g.nh)
    return fail(QEXSTAG_ERR_ARG, "dslash64_ranges: site range outside the parity block");
  DslashArgs64 A;
  std::memset(&A, 0, sizeof(A));
  A.g = g;
  A.po = po;
  A.u = gl->u64;
  A.xin = xin.p;
  A.istride = xin.stride;
  A.xs = xs.p;
  A.sstride = xs.stride;
  A.out = out.p;
  A.ostride = out.stride;
  A.b = b;
  A.c = c;
  A.done = done;
  A.k0 = k0;
  A.n1 = k1 - k0;
  A.k2 = k2;
  A.nsites = (k1 - k0) + (k3 - k2);
  if (A.nsites == 0) return QEXSTAG_OK;
  const int init = xs.p ? 1 : 0;
  const int rc = (gl->nl == 8) ? dispatch64<8>(A, hop, init, kRedNone, grid_for(A.nsites, kBlock, 6))
                               : dispatch64<4>(A, hop, init, kRedNone, grid_for(A.nsites, kBlock, 6));
  if (rc) return rc;
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// One half sweep over nrun runs of rowlen sites of parity po, pitch apart,
// from k0 (a block of z rows in each of a range of t slices): out = b xs +
// c (2D) xin with hop sign hop, no reduction; skipped once *done is set.
int dslash64_rows(const qexstag_links_s *gl, int po, VecD out, CVecD xin, CVecD xs, double b, double c, int hop,
                  int k0, int nrun, int rowlen, int pitch, const int *done) {
  const Geom &g = gl->l->g;
  if (k0 < 0 || nrun < 0 || rowlen < 0 || rowlen > pitch ||
      (nrun > 0 && (long)k0 + (long)(nrun - 1) * pitch + rowlen > g.nh))
    return fail(QEXSTAG_ERR_ARG, "dslash64_rows: site runs outside the parity block");
  DslashArgs64 A;
  std::memset(&A, 0, sizeof(A));
  A.g = g;
  A.po = po;
  A.u = gl->u64;
  A.xin = xin.p;
  A.istride = xin.stride;
  A.xs = xs.p;
  A.sstride = xs.stride;
  A.out = out.p;
  A.ostride = out.stride;
  A.b = b;
  A.c = c;
  A.done = done;
  A.k0 = k0;
  A.rowlen = rowlen;
  A.pitch = pitch;
  A.nsites = nrun * rowlen;
  A.n1 = A.nsites;
  if (A.nsites == 0) return QEXSTAG_OK;
  const int init = xs.p ? 1 : 0;
  const int rc = (gl->nl == 8) ? dispatch64<8>(A, hop, init, kRedNone, grid_for(A.nsites, kBlock, 6))
                               : dispatch64<4>(A, hop, init, kRedNone, grid_for(A.nsites, kBlock, 6));
  if (rc) return rc;
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// stagD2xx (stagD.nim:485-512): t_q = (2D)_{q,par} x (stagDP, rir := 0), then
// r = 4 m2 x - (2D)_{par,q} t (stagDM with rir := 4 m2 x).
int schur64(const qexstag_links_s *gl, int par, VecD r, CVecD x, VecD t, double m2, int red,
            void *state, const int *done, double *dot_out) {
  int rc = dslash64(gl, 1 - par, t, x, CVecD{nullptr, 0}, CVecD{nullptr, 0}, 0.0, 0.0, 1.0, +1,
                    0, kRedNone, nullptr, done);
  if (rc) return rc;
  return dslash64(gl, par, r, cv(t), x, CVecD{nullptr, 0}, 0.0, 4.0 * m2, 1.0, -1, 1, red, state,
                  done, dot_out);
}

}  // namespace qs

namespace qs {

// The FP64 Schur operator with a caller-provided temporary t, launched
// without touching the library's reduction scratch (no reductions, no
// early exit); used by the allocation-free entry point.
int schur64_plain(const qexstag_links_s *gl, int par, VecD r, CVecD x, VecD t, double m2) {
  const Geom &g = gl->l->g;
  DslashArgs64 A;
  std::memset(&A, 0, sizeof(A));
  A.g = g;
  A.u = gl->u64;
  A.n1 = A.nsites = g.nh;
  const int grid = grid_for(g.nh, kBlock, 6);
  // t = (2D)_{q,par} x
  A.po = 1 - par;
  A.xin = x.p;
  A.istride = x.stride;
  A.out = t.p;
  A.ostride = t.stride;
  A.c = 1.0;
  if (gl->nl == 8)
    launch64<8, 1, 0, kRedNone>(A, grid);
  else
    launch64<4, 1, 0, kRedNone>(A, grid);
  // r = 4 m2 x - (2D)_{par,q} t
  A.po = par;
  A.xin = t.p;
  A.istride = t.stride;
  A.xs = x.p;
  A.sstride = x.stride;
  A.out = r.p;
  A.ostride = r.stride;
  A.b = 4.0 * m2;
  if (gl->nl == 8)
    launch64<8, -1, 1, kRedNone>(A, grid);
  else
    launch64<4, -1, 1, kRedNone>(A, grid);
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

}  // namespace qs
