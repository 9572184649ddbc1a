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

// Re det of a Hermitian matrix (cofactors along row 0)
__device__ __forceinline__ double re_det(const M3 &t) {
  const double2 *m = t.e;
  const double2 c0 = make_double2(cmul(m[4], m[8]).x - cmul(m[5], m[7]).x, cmul(m[4], m[8]).y - cmul(m[5], m[7]).y);
  const double2 c1 = make_double2(cmul(m[5], m[6]).x - cmul(m[3], m[8]).x, cmul(m[5], m[6]).y - cmul(m[3], m[8]).y);
  const double2 c2 = make_double2(cmul(m[3], m[7]).x - cmul(m[4], m[6]).x, cmul(m[3], m[7]).y - cmul(m[4], m[6]).y);
  return cmul(m[0], c0).x + cmul(m[1], c1).x + cmul(m[2], c2).x;
}

// W = X (X^dag X + eps)^(-1/2).  The inverse square root of the Hermitian
// H = X^dag X + eps is the quadratic c0 + c1 H + c2 H^2 that takes the value
// 1/sqrt(l) at each eigenvalue l (Cayley-Hamilton); the eigenvalues come from
// the trigonometric solution of the characteristic cubic in tr H, tr H^2 and
// det H, as QEX's projectU does.
__device__ __forceinline__ void project_u(M3 &w, const M3 &x, double eps) {
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
  M3 z;
#pragma unroll
  for (int e = 0; e < 9; e++) z.e[e] = make_double2(c1 * h.e[e].x + c2 * h2.e[e].x, c1 * h.e[e].y + c2 * h2.e[e].y);
  z.e[0].x += c0;
  z.e[4].x += c0;
  z.e[8].x += c0;
  m_nn(w, x, z);
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

static dim3 sweep_grid(const Geom &g) { return dim3((unsigned)(8 * ((g.nh + kSmBlock - 1) / kSmBlock)), 1, 1); }
static dim3 field_grid(const Geom &g) { return dim3((unsigned)((g.V + kSmBlock - 1) / kSmBlock), 4, 1); }

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

// A smearing handle: the layout and the device scratch of the sweeps.
struct qexstag_smear_s {
  qexstag_layout_s *l = nullptr;
  qs::Workspace ws;
};

namespace qs {

enum SmearSlot { kSmS3 = 0, kSmS5, kSmT1, kSmW, kSmIn0, kSmIn1, kSmOut0, kSmOut1, kSmAos };

static size_t field4_bytes(const Geom &g) { return sizeof(double2) * 9 * (size_t)g.V * 4; }

// device view of a 4-direction gauge field given in either memory space
static int smear_in(qexstag_smear_s *s, int slot, const double *p, int mem, const double2 **dev) {
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

static int smear_out_buf(qexstag_smear_s *s, int slot, double *p, int mem, double2 **dev) {
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

static int smear_out_finish(qexstag_smear_s *s, const double2 *dev, double *p, int mem) {
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

static int smear_scratch(qexstag_smear_s *s, const qexstag_fat7_coefs &c, double2 **s3, double2 **s5) {
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

static int check_smear(const qexstag_smear_s *s, int mem) {
  if (!s || !s->l) return fail(QEXSTAG_ERR_ARG, "null or destroyed smearing handle");
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE) return fail(QEXSTAG_ERR_ARG, "bad memory kind");
  return runtime_ready();
}

static bool finite_coefs(const qexstag_fat7_coefs &c) {
  return std::isfinite(c.one_link) && std::isfinite(c.three_staple) && std::isfinite(c.five_staple) &&
         std::isfinite(c.seven_staple) && std::isfinite(c.lepage);
}

// HisqCoefs.smear into device fields fat (stride ffs) and long (stride lfs)
static int hisq_dev(qexstag_smear_s *s, const qexstag_hisq_coefs &c, const double2 *g, double2 *fat, size_t ffs,
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
