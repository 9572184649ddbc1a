// smear.cu -- HISQ link smearing on the device: QEX's makeImpLinks (fat7 with
// Lepage and Naik terms, src/gauge/fat7l.nim:24-154), projectU
// (src/maths/matrixFunctions.nim:118-212, 340-351) and HisqCoefs.smear
// (src/physics/hisqLinks.nim:40-46).
//
// QEX builds the staples field by field: for each (mu, nu) a 3-staple field,
// then Lepage, 5- and 7-staples from shifted copies of it, about 70 field
// sweeps per level.  Here every level takes three sweeps over the lattice,
// one thread per (site, direction mu):
//   sweep 1: S3[mu][nu](x) for the three nu != mu, stored; fl = c1' U + c3 S3
//   sweep 2: Lepage staples of S3 along nu and 5-staples S5[mu][nu][rho]
//            along the two rho not in {mu, nu}, stored; fl += cL L + c5 S5
//   sweep 3: 7-staples of S5 along the remaining direction; fl += c7 S7
// so each staple field is written once and read once from HBM (12 S3 and 24
// S5 fields, 144 B per site each in FP64).  A staple of a field F along nu,
// for the link direction mu, is
//   U_nu(x) F(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag F(x-nu) U_nu(x-nu+mu)
// (computeGenStaple).  The unitary projection and the Naik product
// naik U(x) U(x+mu) U(x+2mu) are one more sweep each.
//
// Fields are double2[4][9][V] (direction, element 3*row+col, site index of
// the QEX V=1 layout), the library's FP64 link layout.
#include "smear.cuh"

namespace qs {

struct Fat7Args {
  Geom g;
  const double2 *u;  // gauge field direction d at u + d*ufs
  size_t ufs;
  double2 *fl;       // fat field direction d at fl + d*ffs
  size_t ffs;
  double2 *s3;       // [4][3][9][V]
  double2 *s5;       // [4][3][2][9][V]
  double c1, c3, c5, c7, cl;
  int have3, store3, do5, store5;
};

// sweep 1: one-link term and 3-staples
__global__ void __launch_bounds__(kSmBlock, 3) fat7_three_kernel(const Fat7Args A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)A.g.V;
  const double2 *Um = A.u + mu * A.ufs;
  M3 acc;
  m_load(acc, Um, V, c.site);
  m_scale(acc, A.c1);
  if (A.have3) {
#pragma unroll 1
    for (int j = 0; j < 3; j++) {
      const int nu = other_dir(mu, j);
      M3 S;
      staple(S, A.g, c, mu, nu, A.u + nu * A.ufs, Um);
      if (A.store3) m_store(A.s3 + (size_t)(mu * 3 + j) * 9 * V, V, c.site, S);
      m_axpy(acc, A.c3, S);
    }
  }
  m_store(A.fl + mu * A.ffs, V, c.site, acc);
}

// sweep 2: Lepage staples and 5-staples of the stored 3-staples
__global__ void __launch_bounds__(kSmBlock, 3) fat7_five_kernel(const Fat7Args A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)A.g.V;
  double2 *flm = A.fl + mu * A.ffs;
  M3 acc;
  m_load(acc, flm, V, c.site);
#pragma unroll 1
  for (int j = 0; j < 3; j++) {
    const int nu = other_dir(mu, j);
    const double2 *F = A.s3 + (size_t)(mu * 3 + j) * 9 * V;
    M3 S;
    if (A.cl != 0.0) {
      staple(S, A.g, c, mu, nu, A.u + nu * A.ufs, F);
      m_axpy(acc, A.cl, S);
    }
    if (A.do5) {
#pragma unroll 1
      for (int r = 0; r < 2; r++) {
        const int rho = third_dir(mu, nu, r);
        staple(S, A.g, c, mu, rho, A.u + rho * A.ufs, F);
        if (A.store5) m_store(A.s5 + (size_t)((mu * 3 + j) * 2 + r) * 9 * V, V, c.site, S);
        m_axpy(acc, A.c5, S);
      }
    }
  }
  m_store(flm, V, c.site, acc);
}

// sweep 3: 7-staples of the stored 5-staples
__global__ void __launch_bounds__(kSmBlock, 3) fat7_seven_kernel(const Fat7Args A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)A.g.V;
  double2 *flm = A.fl + mu * A.ffs;
  M3 acc;
  m_load(acc, flm, V, c.site);
#pragma unroll 1
  for (int j = 0; j < 3; j++) {
    const int nu = other_dir(mu, j);
#pragma unroll 1
    for (int r = 0; r < 2; r++) {
      const int rho = third_dir(mu, nu, r);
      const int sig = 6 - mu - nu - rho;
      M3 S;
      staple(S, A.g, c, mu, sig, A.u + sig * A.ufs, A.s5 + (size_t)((mu * 3 + j) * 2 + r) * 9 * V);
      m_axpy(acc, A.c7, S);
    }
  }
  m_store(flm, V, c.site, acc);
}

// ll_mu(x) = naik U_mu(x) (U_mu(x+mu) U_mu(x+2mu))   (fat7l.nim:142-154)
__global__ void __launch_bounds__(kSmBlock)
    naik_kernel(Geom g, const double2 *__restrict__ u, size_t ufs, double2 *ll, size_t lfs, double naik) {
  SiteCtx c;
  if (!site_of_thread(g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)g.V;
  const double2 *U = u + mu * ufs;
  M3 a, b, t;
  m_load(a, U, V, disp1(g, c.x, c.lex, c.par, mu, 1));
  m_load(b, U, V, disp1(g, c.x, c.lex, c.par, mu, 2));
  m_nn(t, a, b);
  m_load(a, U, V, c.site);
  m_nn(b, a, t);
  m_scale(b, naik);
  m_store(ll + mu * lfs, V, c.site, b);
}

__global__ void __launch_bounds__(kSmBlock)
    project_u_kernel(int V, const double2 *__restrict__ in, size_t ifs, double2 *out, size_t ofs, double eps) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  M3 x, w;
  m_load(x, in + mu * ifs, (size_t)V, s);
  project_u(w, x, eps);
  m_store(out + mu * ofs, (size_t)V, s, w);
}

// makeImpLinks on device fields: u (stride ufs between directions) -> fl
// (stride ffs); s3/s5 scratch
int fat7_dev(const Geom &g, const qexstag_fat7_coefs &c, const double2 *u, size_t ufs, double2 *fl, size_t ffs,
             double2 *s3, double2 *s5) {
  Fat7Args A;
  A.g = g;
  A.u = u;
  A.ufs = ufs;
  A.fl = fl;
  A.ffs = ffs;
  A.s3 = s3;
  A.s5 = s5;
  A.c1 = c.one_link - 6.0 * c.lepage;
  A.c3 = c.three_staple;
  A.c5 = c.five_staple;
  A.c7 = c.seven_staple;
  A.cl = c.lepage;
  const bool have5 = c.five_staple != 0.0 || c.seven_staple != 0.0 || c.lepage != 0.0;
  A.have3 = (c.three_staple != 0.0 || have5) ? 1 : 0;
  A.store3 = have5 ? 1 : 0;
  A.do5 = (c.five_staple != 0.0 || c.seven_staple != 0.0) ? 1 : 0;
  A.store5 = c.seven_staple != 0.0 ? 1 : 0;
  const dim3 grid = sweep_grid(g);
  fat7_three_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
  note_launch();
  if (have5) {
    fat7_five_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
    note_launch();
  }
  if (A.store5) {
    fat7_seven_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
    note_launch();
  }
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

int naik_dev(const Geom &g, const double2 *u, size_t ufs, double2 *ll, size_t lfs, double naik) {
  naik_kernel<<<sweep_grid(g), kSmBlock, 0, stream()>>>(g, u, ufs, ll, lfs, naik);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

int project_u_dev(const Geom &g, const double2 *in, size_t ifs, double2 *out, size_t ofs, double eps) {
  project_u_kernel<<<field_grid(g), kSmBlock, 0, stream()>>>(g.V, in, ifs, out, ofs, eps);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

}  // namespace qs

namespace qs {

// HisqCoefs.smear into device fields fat (stride ffs) and long (stride lfs)
int hisq_dev(qexstag_smear_s *s, const qexstag_hisq_coefs &c, const double2 *g, double2 *fat, size_t ffs,
             double2 *lng, size_t lfs) {
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  void *pt1, *pw;
  double2 *s3, *s5;
  int rc;
  if ((rc = s->ws.get(kSmT1, field4_bytes(geo), &pt1)) || (rc = s->ws.get(kSmW, field4_bytes(geo), &pw))) return rc;
  if ((rc = smear_scratch(s, c.fat7first, &s3, &s5)) ||
      (rc = fat7_dev(geo, c.fat7first, g, fs, (double2 *)pt1, fs, s3, s5)))
    return rc;
  if ((rc = project_u_dev(geo, (const double2 *)pt1, fs, (double2 *)pw, fs, c.reunit_eps))) return rc;
  if ((rc = smear_scratch(s, c.fat7second, &s3, &s5)) ||
      (rc = fat7_dev(geo, c.fat7second, (const double2 *)pw, fs, fat, ffs, s3, s5)))
    return rc;
  if (c.naik != 0.0) return naik_dev(geo, (const double2 *)pw, fs, lng, lfs, c.naik);
  // no Naik term: long links are zero
  for (int d = 0; d < 4; d++) QS_CUDA(cudaMemsetAsync(lng + d * lfs, 0, sizeof(double2) * fs, stream()));
  return QEXSTAG_OK;
}

}  // namespace qs

using namespace qs;

extern "C" {

void qexstag_fat7_coefs_set_hisq(qexstag_fat7_coefs *c, double f7lf, double naik) {
  if (!c) return;
  c->one_link = (1.0 + 3.0 * f7lf + naik) / 8.0;
  c->three_staple = -1.0 / 16.0;
  c->five_staple = 1.0 / 64.0;
  c->seven_staple = -1.0 / 384.0;
  c->lepage = -f7lf / 16.0;
}

void qexstag_hisq_coefs_init(qexstag_hisq_coefs *c, double lepage, double naik) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  qexstag_fat7_coefs_set_hisq(&c->fat7first, lepage, 0.0);
  qexstag_fat7_coefs_set_hisq(&c->fat7second, 2.0 - lepage, naik);
  c->naik = -naik / 24.0;
  c->reunit_eps = 1e-20;
}

int qexstag_smear_create(qexstag_layout *l, qexstag_smear **out) {
  if (!l || !out) return fail(QEXSTAG_ERR_ARG, "smear_create: null argument");
  int rc = runtime_ready();
  if (rc) return rc;
  qexstag_smear_s *s = new (std::nothrow) qexstag_smear_s;
  if (!s) return fail(QEXSTAG_ERR_ALLOC, "smear_create: out of host memory");
  s->l = l;
  *out = s;
  return QEXSTAG_OK;
}

int qexstag_smear_destroy(qexstag_smear *s) {
  if (!s) return QEXSTAG_OK;
  s->ws.release();
  s->l = nullptr;
  delete s;
  return QEXSTAG_OK;
}

int qexstag_fat7(qexstag_smear *s, const qexstag_fat7_coefs *c, const double *gf, double *fl,
                 const double *gf_long, double *ll, double naik, int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!c || !gf || !fl) return fail(QEXSTAG_ERR_ARG, "fat7: null argument");
  if (!finite_coefs(*c) || !std::isfinite(naik)) return fail(QEXSTAG_ERR_ARG, "fat7: coefficients not finite");
  const bool want_long = naik != 0.0 && gf_long && ll;
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  const double2 *u, *ul = nullptr;
  double2 *f, *l = nullptr, *s3, *s5;
  if ((rc = smear_in(s, kSmIn0, gf, mem, &u)) || (rc = smear_out_buf(s, kSmOut0, fl, mem, &f))) return rc;
  if (want_long) {
    if (gf_long == gf)
      ul = u;
    else if ((rc = smear_in(s, kSmIn1, gf_long, mem, &ul)))
      return rc;
    if ((rc = smear_out_buf(s, kSmOut1, ll, mem, &l))) return rc;
  }
  if ((rc = smear_scratch(s, *c, &s3, &s5)) || (rc = fat7_dev(geo, *c, u, fs, f, fs, s3, s5))) return rc;
  if (want_long && (rc = naik_dev(geo, ul, fs, l, fs, naik))) return rc;
  if ((rc = smear_out_finish(s, f, fl, mem))) return rc;
  if (want_long && (rc = smear_out_finish(s, l, ll, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_project_u(qexstag_smear *s, const double *x, double *u, double eps, int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!x || !u) return fail(QEXSTAG_ERR_ARG, "project_u: null argument");
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  const double2 *xin;
  double2 *w;
  if ((rc = smear_in(s, kSmIn0, x, mem, &xin)) || (rc = smear_out_buf(s, kSmOut0, u, mem, &w))) return rc;
  if ((rc = project_u_dev(geo, xin, fs, w, fs, eps)) || (rc = smear_out_finish(s, w, u, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_hisq_smear(qexstag_smear *s, const qexstag_hisq_coefs *c, const double *g, double *fat, double *lng,
                       int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!c || !g || !fat || !lng) return fail(QEXSTAG_ERR_ARG, "hisq_smear: null argument");
  if (!finite_coefs(c->fat7first) || !finite_coefs(c->fat7second) || !std::isfinite(c->naik))
    return fail(QEXSTAG_ERR_ARG, "hisq_smear: coefficients not finite");
  const size_t fs = (size_t)9 * s->l->g.V;
  const double2 *u;
  double2 *f, *l;
  if ((rc = smear_in(s, kSmIn0, g, mem, &u)) || (rc = smear_out_buf(s, kSmOut0, fat, mem, &f)) ||
      (rc = smear_out_buf(s, kSmOut1, lng, mem, &l)))
    return rc;
  if ((rc = hisq_dev(s, *c, u, f, fs, l, fs))) return rc;
  if ((rc = smear_out_finish(s, f, fat, mem)) || (rc = smear_out_finish(s, l, lng, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_hisq(qexstag_links *g, qexstag_smear *s, const qexstag_hisq_coefs *c, const double *thin,
                       int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!g || !g->u64 || !c || !thin) return fail(QEXSTAG_ERR_ARG, "links_hisq: null argument");
  if (g->nl != 8) return fail(QEXSTAG_ERR_ARG, "links_hisq: the link handle must hold 8 (fat+Naik) links");
  if (g->l != s->l) return fail(QEXSTAG_ERR_ARG, "links_hisq: handles on different layouts");
  if (!finite_coefs(c->fat7first) || !finite_coefs(c->fat7second) || !std::isfinite(c->naik))
    return fail(QEXSTAG_ERR_ARG, "links_hisq: coefficients not finite");
  const size_t fs = (size_t)9 * s->l->g.V;
  const double2 *u;
  if ((rc = smear_in(s, kSmIn0, thin, mem, &u))) return rc;
  // fat link of direction mu at list entry 2 mu, long link at 2 mu + 1
  if ((rc = hisq_dev(s, *c, u, g->u64, 2 * fs, g->u64 + fs, 2 * fs))) return rc;
  free_low_links(g->low);
  if ((rc = build_low_links(g))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

}  // extern "C"
