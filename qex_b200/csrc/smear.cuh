// smear.cuh -- device helpers and host plumbing shared by the HISQ smearing
// kernels (smear.cu) and their chain rule (smear_deriv.cu).  Fields are
// double2[4][9][V] (direction, element 3*row+col, site index of the QEX V=1
// layout), the library's FP64 link layout.
#pragma once
#include <cmath>
#include <cstring>
#include <new>

#include "lib.cuh"

namespace qs {

void free_low_links(LowLinks &low);
int build_low_links(qexstag_links_s *g);

constexpr int kSmBlock = 128;

struct M3 {
  double2 e[9];
};

__device__ __forceinline__ void m_load(M3 &m, const double2 *f, size_t V, int s) {
#pragma unroll
  for (int e = 0; e < 9; e++) m.e[e] = __ldg(f + (size_t)e * V + s);
}
__device__ __forceinline__ void m_store(double2 *f, size_t V, int s, const M3 &m) {
#pragma unroll
  for (int e = 0; e < 9; e++) f[(size_t)e * V + s] = m.e[e];
}
__device__ __forceinline__ void m_axpy(M3 &y, double a, const M3 &x) {
#pragma unroll
  for (int e = 0; e < 9; e++) {
    y.e[e].x = fma(a, x.e[e].x, y.e[e].x);
    y.e[e].y = fma(a, x.e[e].y, y.e[e].y);
  }
}
__device__ __forceinline__ void m_scale(M3 &y, double a) {
#pragma unroll
  for (int e = 0; e < 9; e++) {
    y.e[e].x *= a;
    y.e[e].y *= a;
  }
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// r = a b (registers)
__device__ __forceinline__ void m_nn(M3 &r, const M3 &a, const M3 &b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) s = cmadd(s, a.e[3 * i + k], b.e[3 * k + j]);
      r.e[3 * i + j] = s;
    }
}
// r = a^dag b (registers)
__device__ __forceinline__ void m_dn(M3 &r, const M3 &a, const M3 &b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) s = cjmadd(s, a.e[3 * k + i], b.e[3 * k + j]);
      r.e[3 * i + j] = s;
    }
}

// Site index of x + a*mu (periodic): lex moves by the wrapped step, the
// parity flips with a odd (all L even).
// (selects instead of indexing x[] with a runtime direction, which would put
// the coordinates in local memory)
__device__ __forceinline__ int pick(const int v[4], int d) {
  return d == 0 ? v[0] : d == 1 ? v[1] : d == 2 ? v[2] : v[3];
}
// lex offset of moving a steps along mu from coordinate xm (periodic)
__device__ __forceinline__ int lex_step(const Geom &g, const int x[4], int mu, int a) {
  const int xm = pick(x, mu), Lm = pick(g.L, mu);
  int y = xm + a;
  if (y >= Lm) y -= Lm;
  if (y < 0) y += Lm;
  return (y - xm) * pick(g.stride, mu);
}
__device__ __forceinline__ int disp1(const Geom &g, const int x[4], int lex, int par, int mu, int a) {
  const int l = lex + lex_step(g, x, mu, a);
  return (l >> 1) + (((par ^ a) & 1) ? g.nh : 0);
}
// x + a*mu + b*nu, mu != nu
__device__ __forceinline__ int disp2(const Geom &g, const int x[4], int lex, int par, int mu, int a, int nu,
                                     int b) {
  const int l = lex + lex_step(g, x, mu, a) + lex_step(g, x, nu, b);
  return (l >> 1) + (((par ^ a ^ b) & 1) ? g.nh : 0);
}

struct SiteCtx {
  int x[4], lex, par, site, mu;
};

// Block b works on direction b % 4 and parity (b / 4) % 2 of the chunk of
// kSmBlock half-lattice sites b / 8, so the eight blocks that read each
// other's links as neighbours run together and those reads hit L2 (with the
// direction- or parity-major order every link is fetched from HBM again by a
// later pass).
__device__ __forceinline__ bool site_of_thread(const Geom &g, SiteCtx &c) {
  const int b = blockIdx.x;
  c.mu = b & 3;
  c.par = (b >> 2) & 1;
  const int k = (b >> 3) * blockDim.x + threadIdx.x;
  if (k >= g.nh) return false;
  c.site = c.par * g.nh + k;
  site_coords(g, c.par, k, c.x, c.lex);
  return true;
}

// S = U_nu(x) F(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag F(x-nu) U_nu(x-nu+mu).
// Every factor is streamed from memory a row or column at a time, so only
// the partial product t and S are live 3x3 matrices.
__device__ __forceinline__ void staple(M3 &S, const Geom &g, const SiteCtx &c, int mu, int nu,
                                       const double2 *__restrict__ Un, const double2 *__restrict__ F) {
  const size_t V = (size_t)g.V;
  const int s_pn = disp1(g, c.x, c.lex, c.par, nu, 1);
  const int s_pm = disp1(g, c.x, c.lex, c.par, mu, 1);
  const int s_mn = disp1(g, c.x, c.lex, c.par, nu, -1);
  const int s_mnpm = disp2(g, c.x, c.lex, c.par, nu, -1, mu, 1);
  M3 t;
  // upper: t = U_nu(x) F(x+nu) (column k of U times row k of F); S = t U_nu(x+mu)^dag
#pragma unroll
  for (int e = 0; e < 9; e++) t.e[e] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a[3], b[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      a[j] = __ldg(Un + (size_t)(3 * j + k) * V + c.site);
      b[j] = __ldg(F + (size_t)(3 * k + j) * V + s_pn);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) t.e[3 * i + j] = cmadd(t.e[3 * i + j], a[i], b[j]);
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    double2 cr[3];
#pragma unroll
    for (int k = 0; k < 3; k++) cr[k] = __ldg(Un + (size_t)(3 * j + k) * V + s_pm);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) s = cjmadd(s, cr[k], t.e[3 * i + k]);  // conj(c_jk) t_ik
      S.e[3 * i + j] = s;
    }
  }
  // lower: t = U_nu(x-nu)^dag F(x-nu) (rows k of both); S += t U_nu(x-nu+mu)
#pragma unroll
  for (int e = 0; e < 9; e++) t.e[e] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a[3], b[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      a[j] = __ldg(Un + (size_t)(3 * k + j) * V + s_mn);
      b[j] = __ldg(F + (size_t)(3 * k + j) * V + s_mn);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) t.e[3 * i + j] = cjmadd(t.e[3 * i + j], a[i], b[j]);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 cr[3];
#pragma unroll
    for (int j = 0; j < 3; j++) cr[j] = __ldg(Un + (size_t)(3 * k + j) * V + s_mnpm);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) S.e[3 * i + j] = cmadd(S.e[3 * i + j], t.e[3 * i + k], cr[j]);
  }
}

__device__ __forceinline__ int other_dir(int mu, int j) { return j < mu ? j : j + 1; }
// r-th direction (r = 0, 1) not in {mu, nu}
__device__ __forceinline__ int third_dir(int mu, int nu, int r) {
  int d = 0, n = 0;
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (k != mu && k != nu) {
      if (n == r) d = k;
      n++;
    }
  return d;
}

// Re det of a Hermitian matrix (cofactors along row 0)
__device__ __forceinline__ double re_det(const M3 &t) {
  const double2 *m = t.e;
  const double2 c0 = make_double2(cmul(m[4], m[8]).x - cmul(m[5], m[7]).x, cmul(m[4], m[8]).y - cmul(m[5], m[7]).y);
  const double2 c1 = make_double2(cmul(m[5], m[6]).x - cmul(m[3], m[8]).x, cmul(m[5], m[6]).y - cmul(m[3], m[8]).y);
  const double2 c2 = make_double2(cmul(m[3], m[7]).x - cmul(m[4], m[6]).x, cmul(m[3], m[7]).y - cmul(m[4], m[6]).y);
  return cmul(m[0], c0).x + cmul(m[1], c1).x + cmul(m[2], c2).x;
}

// Z = (X^dag X + eps)^(-1/2) and W = X Z.  The inverse square root of the Hermitian
// H = X^dag X + eps is the quadratic c0 + c1 H + c2 H^2 that takes the value
// 1/sqrt(l) at each eigenvalue l (Cayley-Hamilton); the eigenvalues come from
// the trigonometric solution of the characteristic cubic in tr H, tr H^2 and
// det H, as QEX's projectU does.
__device__ __forceinline__ void rsqrt_xdx(M3 &z, const M3 &x, double eps) {
  M3 h, h2;
  m_dn(h, x, x);
  h.e[0].x += eps;
  h.e[4].x += eps;
  h.e[8].x += eps;
  m_nn(h2, h, h);
  const double tr = h.e[0].x + h.e[4].x + h.e[8].x;
  const double p2 = h2.e[0].x + h2.e[4].x + h2.e[8].x;
  const double det = re_det(h);
  const double tr3 = tr * (1.0 / 3.0), tr32 = tr3 * tr3;
  const double q = fabs(0.5 * (p2 * (1.0 / 3.0) - tr32));
  const double r = 0.25 * tr3 * (5.0 * tr32 - p2) - 0.5 * det;
  const double sq = sqrt(q);
  const double isq3 = fmin(3e38, 1.0 / (q * sq));
  const double rs = fmax(-1.0, fmin(1.0, r * isq3));
  const double th = acos(rs) * (1.0 / 3.0);
  double st, ct;
  sincos(th, &st, &ct);
  const double sqc = sq * ct, sqs = 1.7320508075688772 * sq * st;
  const double l0 = tr3 - 2.0 * sqc, l1 = tr3 + sqc + sqs, l2 = tr3 + sqc - sqs;
  const double s0 = sqrt(fabs(l0)), s1 = sqrt(fabs(l1)), s2 = sqrt(fabs(l2));
  const double us = s0 + s1 + s2, ws = s0 * s1 * s2;
  const double di = 1.0 / (ws * (s0 + s1) * (s0 + s2) * (s1 + s2));
  const double c0 = (ws * us * us + l0 * s0 * (l1 + l2) + l1 * s1 * (l0 + l2) + l2 * s2 * (l0 + l1)) * di;
  const double c1 = -(tr * us + ws) * di, c2 = us * di;
#pragma unroll
  for (int e = 0; e < 9; e++) z.e[e] = make_double2(c1 * h.e[e].x + c2 * h2.e[e].x, c1 * h.e[e].y + c2 * h2.e[e].y);
  z.e[0].x += c0;
  z.e[4].x += c0;
  z.e[8].x += c0;
}
__device__ __forceinline__ void project_u(M3 &w, const M3 &x, double eps) {
  M3 z;
  rsqrt_xdx(z, x, eps);
  m_nn(w, x, z);
}

inline dim3 sweep_grid(const Geom &g) { return dim3((unsigned)(8 * ((g.nh + kSmBlock - 1) / kSmBlock)), 1, 1); }
inline dim3 field_grid(const Geom &g) { return dim3((unsigned)((g.V + kSmBlock - 1) / kSmBlock), 4, 1); }

// makeImpLinks on device fields: u (stride ufs between directions) -> fl
// (stride ffs); s3 ([4][3][9][V]) and s5 ([4][3][2][9][V]) receive the 3- and
// 5-staples
int fat7_dev(const Geom &g, const qexstag_fat7_coefs &c, const double2 *u, size_t ufs, double2 *fl, size_t ffs,
             double2 *s3, double2 *s5);
int naik_dev(const Geom &g, const double2 *u, size_t ufs, double2 *ll, size_t lfs, double naik);
int project_u_dev(const Geom &g, const double2 *in, size_t ifs, double2 *out, size_t ofs, double eps);

}  // namespace qs

// A smearing handle: the layout and the device scratch of the sweeps.
struct qexstag_smear_s {
  qexstag_layout_s *l = nullptr;
  qs::Workspace ws;
};

namespace qs {

enum SmearSlot { kSmS3 = 0, kSmS5, kSmT1, kSmW, kSmIn0, kSmIn1, kSmOut0, kSmOut1, kSmAos };

inline size_t field4_bytes(const Geom &g) { return sizeof(double2) * 9 * (size_t)g.V * 4; }

// device view of a 4-direction gauge field given in either memory space
inline int smear_in(qexstag_smear_s *s, int slot, const double *p, int mem, const double2 **dev) {
  const Geom &g = s->l->g;
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (const double2 *)p;
    return QEXSTAG_OK;
  }
  void *soa, *aos;
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  int rc;
  if ((rc = s->ws.get(slot, 4 * per, &soa)) || (rc = s->ws.get(kSmAos, per, &aos))) return rc;
  for (int d = 0; d < 4; d++) {
    QS_CUDA(cudaMemcpyAsync(aos, p + (size_t)d * 18 * g.V, per, cudaMemcpyHostToDevice, stream()));
    if ((rc = aos_to_soa((const double *)aos, (double2 *)soa + (size_t)d * 9 * g.V, g.V, g.V, 9))) return rc;
  }
  *dev = (const double2 *)soa;
  return QEXSTAG_OK;
}

inline int smear_out_buf(qexstag_smear_s *s, int slot, double *p, int mem, double2 **dev) {
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (double2 *)p;
    return QEXSTAG_OK;
  }
  void *soa;
  int rc = s->ws.get(slot, field4_bytes(s->l->g), &soa);
  if (rc) return rc;
  *dev = (double2 *)soa;
  return QEXSTAG_OK;
}

inline int smear_out_finish(qexstag_smear_s *s, const double2 *dev, double *p, int mem) {
  if (mem == QEXSTAG_MEM_DEVICE) return QEXSTAG_OK;
  const Geom &g = s->l->g;
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  void *aos;
  int rc = s->ws.get(kSmAos, per, &aos);
  if (rc) return rc;
  for (int d = 0; d < 4; d++) {
    if ((rc = soa_to_aos(dev + (size_t)d * 9 * g.V, (double *)aos, g.V, g.V, 9))) return rc;
    QS_CUDA(cudaMemcpyAsync(p + (size_t)d * 18 * g.V, aos, per, cudaMemcpyDeviceToHost, stream()));
  }
  return QEXSTAG_OK;
}

inline int smear_scratch(qexstag_smear_s *s, const qexstag_fat7_coefs &c, double2 **s3, double2 **s5) {
  const Geom &g = s->l->g;
  const size_t f = sizeof(double2) * 9 * (size_t)g.V;
  void *p3 = nullptr, *p5 = nullptr;
  int rc;
  const bool have5 = c.five_staple != 0.0 || c.seven_staple != 0.0 || c.lepage != 0.0;
  if (have5 && (rc = s->ws.get(kSmS3, 12 * f, &p3))) return rc;
  if (c.seven_staple != 0.0 && (rc = s->ws.get(kSmS5, 24 * f, &p5))) return rc;
  *s3 = (double2 *)p3;
  *s5 = (double2 *)p5;
  return QEXSTAG_OK;
}

inline int check_smear(const qexstag_smear_s *s, int mem) {
  if (!s || !s->l) return fail(QEXSTAG_ERR_ARG, "null or destroyed smearing handle");
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE) return fail(QEXSTAG_ERR_ARG, "bad memory kind");
  return runtime_ready();
}

inline bool finite_coefs(const qexstag_fat7_coefs &c) {
  return std::isfinite(c.one_link) && std::isfinite(c.three_staple) && std::isfinite(c.five_staple) &&
         std::isfinite(c.seven_staple) && std::isfinite(c.lepage);
}

// HisqCoefs.smear of device links g into fat (stride ffs) and long (stride lfs)
int hisq_dev(qexstag_smear_s *s, const qexstag_hisq_coefs &c, const double2 *g, double2 *fat, size_t ffs,
             double2 *lng, size_t lfs);

}  // namespace qs
