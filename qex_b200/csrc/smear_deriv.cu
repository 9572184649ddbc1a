// smear_deriv.cu -- the chain rule through HISQ smearing on the device: the
// derivative of S = sum_x Re Tr C(x)^dag out(x) with respect to the input
// links, in QEX's convention dS = sum Re Tr dU^dag f
// (src/gauge/hisqsmear.nim:66-168: smearGetForce and its check).  QEX
// computes it as fat7lDeriv (src/gauge/fat7lderiv.nim:122-331), projectUderiv
// (src/maths/matrixFunctions.nim:368-390) and fat7lDeriv again.
//
// Here each fat7 level is differentiated in three gather sweeps over
// (site, direction), with the level's 3- and 5-staple fields S3, S5 from a
// forward sweep (smear.cu).  With M the chain on the fat links:
//   sweep A: T7[mu][sig] = St(U_sig; M_mu)        (chain of the 7-staples on
//            the 5-staples, up to c7: M5[mu][nu][rho] = c5 M_mu + c7 T7[mu][sig])
//   sweep B: M3[mu][nu] = c3 M_mu + cL T7[mu][nu] + sum_rho St(U_rho; M5)
//            (chain on the 3-staples)
//   sweep C: dU_d(y) = c1' M_d + sum_nu St(U_nu; M3[d][nu])   (U_d as the
//            middle link of its 3-staples) + the derivatives of every staple
//            in which U_d is a side link: 3-staples (chain M3), Lepage (cL M,
//            middle S3), 5-staples (M5, middle S3), 7-staples (c7 M, middle S5)
//            + the Naik product's three positions.
// St(g; F) = g(x) F(x+nu) g(x+mu)^dag + g(x-nu)^dag F(x-nu) g(x-nu+mu) is the
// staple of the field F along nu; it is also its own adjoint in F, which is
// why the chains on the inner staples are staples of the outer chains.  The
// derivative of St(g1; g2) (side direction d1, link direction d2) with chain c
// with respect to the side field at y is
//   c(y) g1(y+d2) g2(y+d1)^dag + g2(y) g1(y+d2) c(y+d1)^dag
//   + c(y-d2)^dag g1(y-d2) g2(y-d2+d1) + g2(y-d2)^dag g1(y-d2) c(y-d2+d1),
// so every derivative is gathered at its own site: no atomics, no scatter.
#include "smear.cuh"

namespace qs {

// r = a b^dag (registers)
__device__ __forceinline__ void m_nd(M3 &r, const M3 &a, const M3 &b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) s = cjmadd(s, b.e[3 * j + k], a.e[3 * i + k]);
      r.e[3 * i + j] = s;
    }
}

// a field operand sum_k c_k F_k of N fields, element e of site s at e*V + s;
// terms with a zero coefficient are skipped (their pointer may be null)
template <int N>
struct Lin {
  const double2 *p[N];
  double c[N];
  __device__ __forceinline__ double2 ld(size_t o) const {
    double2 r = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < N; k++)
      if (c[k] != 0.0) {
        const double2 x = __ldg(p[k] + o);
        r.x = fma(c[k], x.x, r.x);
        r.y = fma(c[k], x.y, r.y);
      }
    return r;
  }
};
__device__ __forceinline__ Lin<1> lin(const double2 *a, double ca = 1.0) {
  Lin<1> l;
  l.p[0] = a;
  l.c[0] = ca;
  return l;
}

// acc += coef (A B) C^dag; operands streamed a column / row at a time
template <class FA, class FB, class FC>
__device__ __forceinline__ void acc_nn_nd(M3 &acc, double coef, const FA &A, int sa, const FB &B, int sb,
                                          const FC &C, int sc, size_t V) {
  M3 t;
#pragma unroll
  for (int e = 0; e < 9; e++) t.e[e] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a[3], b[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      a[j] = A.ld((size_t)(3 * j + k) * V + sa);
      b[j] = B.ld((size_t)(3 * k + j) * V + sb);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) t.e[3 * i + j] = cmadd(t.e[3 * i + j], a[i], b[j]);
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    double2 c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) c[k] = C.ld((size_t)(3 * j + k) * V + sc);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) s = cjmadd(s, c[k], t.e[3 * i + k]);
      acc.e[3 * i + j].x = fma(coef, s.x, acc.e[3 * i + j].x);
      acc.e[3 * i + j].y = fma(coef, s.y, acc.e[3 * i + j].y);
    }
  }
}

// acc += coef (A^dag B) C
template <class FA, class FB, class FC>
__device__ __forceinline__ void acc_dn_nn(M3 &acc, double coef, const FA &A, int sa, const FB &B, int sb,
                                          const FC &C, int sc, size_t V) {
  M3 t;
#pragma unroll
  for (int e = 0; e < 9; e++) t.e[e] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 a[3], b[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      a[j] = A.ld((size_t)(3 * k + j) * V + sa);
      b[j] = B.ld((size_t)(3 * k + j) * V + sb);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) t.e[3 * i + j] = cjmadd(t.e[3 * i + j], a[i], b[j]);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 c[3];
#pragma unroll
    for (int j = 0; j < 3; j++) c[j] = C.ld((size_t)(3 * k + j) * V + sc);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const double2 tik = make_double2(coef * t.e[3 * i + k].x, coef * t.e[3 * i + k].y);
#pragma unroll
      for (int j = 0; j < 3; j++) acc.e[3 * i + j] = cmadd(acc.e[3 * i + j], tik, c[j]);
    }
  }
}

// acc += coef St(g; F) for link direction mu, staple direction nu
template <class FF>
__device__ __forceinline__ void staple_acc(M3 &acc, double coef, const Geom &g, const SiteCtx &c, int mu, int nu,
                                           const double2 *Un, const FF &F) {
  const size_t V = (size_t)g.V;
  const Lin<1> U = lin(Un);
  const int s_pn = disp1(g, c.x, c.lex, c.par, nu, 1);
  const int s_pm = disp1(g, c.x, c.lex, c.par, mu, 1);
  const int s_mn = disp1(g, c.x, c.lex, c.par, nu, -1);
  const int s_mnpm = disp2(g, c.x, c.lex, c.par, nu, -1, mu, 1);
  acc_nn_nd(acc, coef, U, c.site, F, s_pn, U, s_pm, V);
  acc_dn_nn(acc, coef, U, s_mn, F, s_mn, U, s_mnpm, V);
}

// acc += coef d/dg1 [chain c on St(g1; g2)] at y, g1 the side field of this
// thread's direction d (= d1), g2 of link direction d2
template <class F2, class FC>
__device__ __forceinline__ void side_acc(M3 &acc, double coef, const Geom &g, const SiteCtx &c, int d, int d2,
                                         const double2 *G1, const F2 &G2, const FC &C) {
  const size_t V = (size_t)g.V;
  const Lin<1> g1 = lin(G1);
  const int s_p2 = disp1(g, c.x, c.lex, c.par, d2, 1);
  const int s_p1 = disp1(g, c.x, c.lex, c.par, d, 1);
  const int s_m2 = disp1(g, c.x, c.lex, c.par, d2, -1);
  const int s_m2p1 = disp2(g, c.x, c.lex, c.par, d2, -1, d, 1);
  acc_nn_nd(acc, coef, C, c.site, g1, s_p2, G2, s_p1, V);
  acc_nn_nd(acc, coef, G2, c.site, g1, s_p2, C, s_p1, V);
  acc_dn_nn(acc, coef, C, s_m2, g1, s_m2, G2, s_m2p1, V);
  acc_dn_nn(acc, coef, G2, s_m2, g1, s_m2, C, s_m2p1, V);
}

struct AdjArgs {
  Geom g;
  const double2 *u;   // level input links, direction d at u + d*ufs
  size_t ufs;
  const double2 *m;   // chain on the fat links, stride mfs
  size_t mfs;
  const double2 *lm;  // chain on the long links (nullptr: no Naik term), stride lmfs
  size_t lmfs;
  double naik;
  const double2 *s3;  // [4][3][9][V] forward 3-staples (nullptr when the level has none)
  const double2 *s5;  // [4][3][2][9][V] forward 5-staples (when c7 != 0)
  double2 *t7;        // [4][3][9][V] St(U_sig; M_mu), sig = other_dir(mu, k)
  double2 *m3;        // [4][3][9][V] chain on the 3-staples
  double2 *d;         // output derivative, stride dfs
  size_t dfs;
  int accumulate;     // add to d instead of overwriting it
  double c1, c3, c5, c7, cl;
  int have3, have5, do5;
};

__device__ __forceinline__ size_t fld(const Geom &g, int k) { return (size_t)k * 9 * g.V; }
// index j of direction d among the three directions other than mu
__device__ __forceinline__ int other_index(int mu, int d) { return d < mu ? d : d - 1; }
// index r of rho among the two directions other than mu and nu
__device__ __forceinline__ int third_index(int mu, int nu, int rho) { return rho < 6 - mu - nu - rho ? 0 : 1; }

// sweep A: T7[mu][k] = St(U_sig; M_mu), sig = other_dir(mu, k)
__global__ void __launch_bounds__(kSmBlock, 3) fat7_adj_seven_kernel(const AdjArgs A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)A.g.V;
  const Lin<1> M = lin(A.m + mu * A.mfs);
#pragma unroll 1
  for (int k = 0; k < 3; k++) {
    const int sig = other_dir(mu, k);
    M3 S;
#pragma unroll
    for (int e = 0; e < 9; e++) S.e[e] = make_double2(0.0, 0.0);
    staple_acc(S, 1.0, A.g, c, mu, sig, A.u + sig * A.ufs, M);
    m_store(A.t7 + fld(A.g, mu * 3 + k), V, c.site, S);
  }
}

// sweep B: M3[mu][j] = c3 M_mu + cL St(U_nu; M_mu) + sum_rho St(U_rho; M5[mu][nu][rho]).
// St(U_x; M_mu) is T7[mu][x], so only the c7 part of M5 needs new staples:
//   M3 = c3 M + cL T7[mu][nu] + sum_rho (c5 T7[mu][rho] + c7 St(U_rho; T7[mu][sig]))
__global__ void __launch_bounds__(kSmBlock, 3) fat7_adj_three_kernel(const AdjArgs A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)A.g.V;
  const double2 *Mm = A.m + mu * A.mfs;
#pragma unroll 1
  for (int j = 0; j < 3; j++) {
    const int nu = other_dir(mu, j);
    M3 S, t;
    m_load(S, Mm, V, c.site);
    m_scale(S, A.c3);
    if (A.cl != 0.0) {
      m_load(t, A.t7 + fld(A.g, mu * 3 + j), V, c.site);
      m_axpy(S, A.cl, t);
    }
    if (A.do5) {
#pragma unroll 1
      for (int r = 0; r < 2; r++) {
        const int rho = third_dir(mu, nu, r);
        const int sig = 6 - mu - nu - rho;
        if (A.c5 != 0.0) {
          m_load(t, A.t7 + fld(A.g, mu * 3 + other_index(mu, rho)), V, c.site);
          m_axpy(S, A.c5, t);
        }
        if (A.c7 != 0.0)
          staple_acc(S, A.c7, A.g, c, mu, rho, A.u + rho * A.ufs, lin(A.t7 + fld(A.g, mu * 3 + other_index(mu, sig))));
      }
    }
    m_store(A.m3 + fld(A.g, mu * 3 + j), V, c.site, S);
  }
}

// sweep C: the derivative with respect to U_d at y
__global__ void __launch_bounds__(kSmBlock, 3) fat7_adj_link_kernel(const AdjArgs A) {
  SiteCtx c;
  if (!site_of_thread(A.g, c)) return;
  const int d = c.mu;
  const Geom &g = A.g;
  const size_t V = (size_t)g.V;
  const double2 *Ud = A.u + d * A.ufs;
  M3 acc;
  if (A.accumulate) {
    m_load(acc, A.d + d * A.dfs, V, c.site);
  } else {
#pragma unroll
    for (int e = 0; e < 9; e++) acc.e[e] = make_double2(0.0, 0.0);
  }
  {
    M3 md;
    m_load(md, A.m + d * A.mfs, V, c.site);
    m_axpy(acc, A.c1, md);
  }
  if (A.have3) {
    // U_d as the middle link of its 3-staples
#pragma unroll 1
    for (int j = 0; j < 3; j++) {
      const int nu = other_dir(d, j);
      staple_acc(acc, 1.0, g, c, d, nu, A.u + nu * A.ufs, lin(A.m3 + fld(g, d * 3 + j)));
    }
    // U_d as a side link.  A side derivative is linear in its middle field
    // and in its chain, so the terms with chain M_mu are taken together:
    // Lepage (cL, middle S3[mu][d]), the c5 part of the 5-staples (middle
    // S3[mu][nu]) and the 7-staples (c7, middle S5[mu][nu][rho]).
#pragma unroll 1
    for (int jm = 0; jm < 3; jm++) {
      const int mu = other_dir(d, jm);
      const int jd = other_index(mu, d);
      const double2 *Mm = A.m + mu * A.mfs;
      // 3-staple S3[mu][d] = St(U_d; U_mu), chain M3[mu][d]
      side_acc(acc, 1.0, g, c, d, mu, Ud, lin(A.u + mu * A.ufs), lin(A.m3 + fld(g, mu * 3 + jd)));
      if (A.have5) {
        const int nu0 = third_dir(mu, d, 0), nu1 = third_dir(mu, d, 1);
        const int jn0 = other_index(mu, nu0), jn1 = other_index(mu, nu1);
        const int rho0 = 6 - mu - nu0 - d, rho1 = 6 - mu - nu1 - d;  // the fourth directions
        Lin<5> G;
        G.p[0] = A.s3 + fld(g, mu * 3 + jd);
        G.c[0] = A.cl;
        G.p[1] = A.s3 + fld(g, mu * 3 + jn0);
        G.c[1] = A.c5;
        G.p[2] = A.s3 + fld(g, mu * 3 + jn1);
        G.c[2] = A.c5;
        G.p[3] = A.c7 != 0.0 ? A.s5 + fld(g, (mu * 3 + jn0) * 2 + third_index(mu, nu0, rho0)) : nullptr;
        G.c[3] = A.c7;
        G.p[4] = A.c7 != 0.0 ? A.s5 + fld(g, (mu * 3 + jn1) * 2 + third_index(mu, nu1, rho1)) : nullptr;
        G.c[4] = A.c7;
        side_acc(acc, 1.0, g, c, d, mu, Ud, G, lin(Mm));
        // the c7 part of the 5-staple chains M5[mu][nu][d] = c5 M_mu + c7 T7[mu][rho]
        if (A.c7 != 0.0) {
          side_acc(acc, A.c7, g, c, d, mu, Ud, lin(A.s3 + fld(g, mu * 3 + jn0)),
                   lin(A.t7 + fld(g, mu * 3 + other_index(mu, rho0))));
          side_acc(acc, A.c7, g, c, d, mu, Ud, lin(A.s3 + fld(g, mu * 3 + jn1)),
                   lin(A.t7 + fld(g, mu * 3 + other_index(mu, rho1))));
        }
      }
    }
  }
  if (A.lm) {
    // ll_d(x) = naik W(x) W(x+d) W(x+2d), W = U_d: the three positions of y
    const double2 *LM = A.lm + d * A.lmfs;
    const int s_p1 = disp1(g, c.x, c.lex, c.par, d, 1), s_p2 = disp1(g, c.x, c.lex, c.par, d, 2);
    const int s_m1 = disp1(g, c.x, c.lex, c.par, d, -1), s_m2 = disp1(g, c.x, c.lex, c.par, d, -2);
    M3 a, b, t;
    // LM(y) (W(y+d) W(y+2d))^dag
    m_load(a, Ud, V, s_p1);
    m_load(b, Ud, V, s_p2);
    m_nn(t, a, b);
    m_load(a, LM, V, c.site);
    m_nd(b, a, t);
    m_axpy(acc, A.naik, b);
    // W(y-d)^dag LM(y-d) W(y+d)^dag
    m_load(a, Ud, V, s_m1);
    m_load(b, LM, V, s_m1);
    m_dn(t, a, b);
    m_load(a, Ud, V, s_p1);
    m_nd(b, t, a);
    m_axpy(acc, A.naik, b);
    // (W(y-2d) W(y-d))^dag LM(y-2d)
    m_load(a, Ud, V, s_m2);
    m_load(b, Ud, V, s_m1);
    m_nn(t, a, b);
    m_load(a, LM, V, s_m2);
    m_dn(b, t, a);
    m_axpy(acc, A.naik, b);
  }
  m_store(A.d + d * A.dfs, V, c.site, acc);
}

// ---------------------------------------------------------------------------
// projectU's chain rule (matrixFunctions.nim:368-390): U = X Z, Z = (X^dag X +
// eps)^(-1/2), Y = Z^-1; with chain C
//   r = C Z - X (T + T^dag),   Y T + T Y = U^dag C Z
// The Sylvester equation is solved in closed form from the adjugate and the
// invariants of Y (projUderiv.nim:96-145, 3x3 branch).
// ---------------------------------------------------------------------------

__device__ __forceinline__ void m_adjugate(M3 &r, const M3 &x) {
  const double2 *m = x.e;
  auto sub = [](double2 a, double2 b, double2 c, double2 d) {
    const double2 p = cmul(a, b), q = cmul(c, d);
    return make_double2(p.x - q.x, p.y - q.y);
  };
  r.e[0] = sub(m[4], m[8], m[5], m[7]);
  r.e[1] = sub(m[7], m[2], m[8], m[1]);
  r.e[2] = sub(m[1], m[5], m[2], m[4]);
  r.e[3] = sub(m[5], m[6], m[3], m[8]);
  r.e[4] = sub(m[8], m[0], m[6], m[2]);
  r.e[5] = sub(m[2], m[3], m[0], m[5]);
  r.e[6] = sub(m[3], m[7], m[4], m[6]);
  r.e[7] = sub(m[6], m[1], m[7], m[0]);
  r.e[8] = sub(m[0], m[4], m[1], m[3]);
}

// x with a x + x a = c, a Hermitian positive definite (invariants real)
__device__ __forceinline__ void sylsolve3(M3 &x, const M3 &a, const M3 &c) {
  M3 ad, p, q;
  m_adjugate(ad, a);
  const double t = a.e[0].x + a.e[4].x + a.e[8].x;
  const double s = ad.e[0].x + ad.e[4].x + ad.e[8].x;
  const double r = cmul(a.e[0], ad.e[0]).x + cmul(a.e[1], ad.e[3]).x + cmul(a.e[2], ad.e[6]).x;
  const double c2 = 1.0 / (2.0 * (s * t - r));
  const double c0 = c2 * (s + t * t), c1 = c2 * (t / r), c4 = c2 * t;
#pragma unroll
  for (int e = 0; e < 9; e++) x.e[e] = make_double2(c0 * c.e[e].x, c0 * c.e[e].y);
  m_nn(p, a, c);       // a c
  m_axpy(x, -c4, p);
  m_nn(q, p, a);       // a c a
  m_axpy(x, c2, q);
  m_nn(p, c, a);       // c a
  m_axpy(x, -c4, p);
  m_nn(p, ad, c);      // ad c
  m_axpy(x, -c2, p);
  m_nn(q, p, ad);      // ad c ad
  m_axpy(x, c1, q);
  m_nn(p, c, ad);      // c ad
  m_axpy(x, -c2, p);
}

__global__ void __launch_bounds__(kSmBlock)
    project_u_deriv_kernel(int V, const double2 *__restrict__ u, const double2 *__restrict__ x,
                           const double2 *chain, double2 *out, size_t fs, double eps) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t off = blockIdx.y * fs;
  M3 X, Z, Y, R, T;
  m_load(X, x + off, (size_t)V, s);
  rsqrt_xdx(Z, X, eps);
  {
    // Y = Z^-1 = adj(Z) / det Z
    M3 ad;
    m_adjugate(ad, Z);
    const double2 det = make_double2(cmul(Z.e[0], ad.e[0]).x + cmul(Z.e[1], ad.e[3]).x + cmul(Z.e[2], ad.e[6]).x,
                                     cmul(Z.e[0], ad.e[0]).y + cmul(Z.e[1], ad.e[3]).y + cmul(Z.e[2], ad.e[6]).y);
    const double nn = det.x * det.x + det.y * det.y;
    const double2 idet = make_double2(det.x / nn, -det.y / nn);
#pragma unroll
    for (int e = 0; e < 9; e++) Y.e[e] = cmul(ad.e[e], idet);
  }
  m_load(T, chain + off, (size_t)V, s);
  m_nn(R, T, Z);  // C Z
  m_load(T, u + off, (size_t)V, s);
  m_dn(Z, T, R);  // U^dag C Z
  sylsolve3(T, Y, Z);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double2 a = T.e[3 * i + j], b = T.e[3 * j + i];
      Z.e[3 * i + j] = make_double2(a.x + b.x, a.y - b.y);  // T + T^dag
    }
  m_nn(T, X, Z);
  m_axpy(R, -1.0, T);
  m_store(out + off, (size_t)V, s, R);
}

int project_u_deriv_dev(const Geom &g, const double2 *u, const double2 *x, const double2 *chain, double2 *out,
                        double eps) {
  project_u_deriv_kernel<<<field_grid(g), kSmBlock, 0, stream()>>>(g.V, u, x, chain, out, (size_t)9 * g.V, eps);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// fat7lDeriv on device fields: d (+)= derivative w.r.t. u of
// sum Re Tr (m^dag fat7(u) + lm^dag naik u(x)u(x+mu)u(x+2mu)); s3/s5 hold the
// level's forward staples (fat7_dev on u), t7 and m3 are 12-field scratch.
int fat7_adj_dev(const Geom &g, const qexstag_fat7_coefs &c, const double2 *u, size_t ufs, const double2 *m,
                 size_t mfs, const double2 *lm, size_t lmfs, double naik, const double2 *s3, const double2 *s5,
                 double2 *t7, double2 *m3, double2 *d, size_t dfs, bool accumulate) {
  AdjArgs A;
  A.g = g;
  A.u = u;
  A.ufs = ufs;
  A.m = m;
  A.mfs = mfs;
  A.lm = (naik != 0.0) ? lm : nullptr;
  A.lmfs = lmfs;
  A.naik = naik;
  A.s3 = s3;
  A.s5 = s5;
  A.t7 = t7;
  A.m3 = m3;
  A.d = d;
  A.dfs = dfs;
  A.accumulate = accumulate ? 1 : 0;
  A.c1 = c.one_link - 6.0 * c.lepage;
  A.c3 = c.three_staple;
  A.c5 = c.five_staple;
  A.c7 = c.seven_staple;
  A.cl = c.lepage;
  A.have5 = (c.five_staple != 0.0 || c.seven_staple != 0.0 || c.lepage != 0.0) ? 1 : 0;
  A.have3 = (c.three_staple != 0.0 || A.have5) ? 1 : 0;
  A.do5 = (c.five_staple != 0.0 || c.seven_staple != 0.0) ? 1 : 0;
  const dim3 grid = sweep_grid(g);
  if (A.have5) {
    fat7_adj_seven_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
    note_launch();
  }
  if (A.have3) {
    fat7_adj_three_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
    note_launch();
  }
  fat7_adj_link_kernel<<<grid, kSmBlock, 0, stream()>>>(A);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

enum DerivSlot { kSdT7 = 40, kSdM3, kSdV, kSdW, kSdTmp, kSdDW, kSdIn2, kSdIn3, kSdOut2 };

static int adj_scratch(qexstag_smear_s *s, double2 **t7, double2 **m3) {
  const size_t f = sizeof(double2) * 9 * (size_t)s->l->g.V;
  void *a, *b;
  int rc;
  if ((rc = s->ws.get(kSdT7, 12 * f, &a)) || (rc = s->ws.get(kSdM3, 12 * f, &b))) return rc;
  *t7 = (double2 *)a;
  *m3 = (double2 *)b;
  return QEXSTAG_OK;
}

// smearGetForce's chain rule on device fields
static int hisq_deriv_dev(qexstag_smear_s *s, const qexstag_hisq_coefs &c, const double2 *g, const double2 *cf,
                          size_t cfs, const double2 *cl, size_t cls, double2 *d) {
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  void *pv, *pw, *pt, *pd;
  double2 *s3, *s5, *t7, *m3;
  int rc;
  if ((rc = s->ws.get(kSdV, field4_bytes(geo), &pv)) || (rc = s->ws.get(kSdW, field4_bytes(geo), &pw)) ||
      (rc = s->ws.get(kSdTmp, field4_bytes(geo), &pt)) || (rc = s->ws.get(kSdDW, field4_bytes(geo), &pd)) ||
      (rc = adj_scratch(s, &t7, &m3)))
    return rc;
  double2 *v = (double2 *)pv, *w = (double2 *)pw, *tmp = (double2 *)pt, *dw = (double2 *)pd;
  // forward: v = fat7(g), w = projectU(v), and the second level's staples
  if ((rc = smear_scratch(s, c.fat7first, &s3, &s5)) || (rc = fat7_dev(geo, c.fat7first, g, fs, v, fs, s3, s5)) ||
      (rc = project_u_dev(geo, v, fs, w, fs, c.reunit_eps)) || (rc = smear_scratch(s, c.fat7second, &s3, &s5)) ||
      (rc = fat7_dev(geo, c.fat7second, w, fs, tmp, fs, s3, s5)))
    return rc;
  // second level (fat7 and Naik both of w) -> dS/dw
  if ((rc = fat7_adj_dev(geo, c.fat7second, w, fs, cf, cfs, cl, cls, c.naik, s3, s5, t7, m3, dw, fs, false)))
    return rc;
  // projectU -> dS/dv (in place)
  if ((rc = project_u_deriv_dev(geo, w, v, dw, dw, c.reunit_eps))) return rc;
  // first level: its staples again, then dS/dg
  if ((rc = smear_scratch(s, c.fat7first, &s3, &s5)) || (rc = fat7_dev(geo, c.fat7first, g, fs, tmp, fs, s3, s5)))
    return rc;
  return fat7_adj_dev(geo, c.fat7first, g, fs, dw, fs, nullptr, 0, 0.0, s3, s5, t7, m3, d, fs, false);
}

// F_d(x) = projectTAH(ff_d(x) U_d(x)^dag)   (fermForce's last step,
// hmcAction.nim:780-790; projectTAH: matrixFunctions.nim:414-419)
__global__ void __launch_bounds__(kSmBlock)
    tah_times_adj_kernel(int V, const double2 *__restrict__ ff, const double2 *__restrict__ u, double2 *out,
                         size_t fs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t off = blockIdx.y * fs;
  M3 a, b, m;
  m_load(a, ff + off, (size_t)V, s);
  m_load(b, u + off, (size_t)V, s);
  m_nd(m, a, b);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double2 p = m.e[3 * i + j], q = m.e[3 * j + i];
      a.e[3 * i + j] = make_double2(0.5 * (p.x - q.x), 0.5 * (p.y + q.y));
    }
  const double tr = (a.e[0].y + a.e[4].y + a.e[8].y) * (1.0 / 3.0);
  a.e[0].y -= tr;
  a.e[4].y -= tr;
  a.e[8].y -= tr;
  m_store(out + off, (size_t)V, s, a);
}

enum ForceSlot { kSfPhi = 60, kSfPsi, kSfF8, kSfFF };

}  // namespace qs

using namespace qs;

extern "C" {

int qexstag_fat7_deriv(qexstag_smear *s, const qexstag_fat7_coefs *c, const double *gauge, const double *mid,
                       double *deriv, const double *llgauge, const double *llmid, double *llderiv, double naik,
                       int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!c || !gauge || !mid || !deriv) return fail(QEXSTAG_ERR_ARG, "fat7_deriv: null argument");
  if (!finite_coefs(*c) || !std::isfinite(naik)) return fail(QEXSTAG_ERR_ARG, "fat7_deriv: coefficients not finite");
  const bool want_long = naik != 0.0 && llgauge && llmid && llderiv;
  const bool same = want_long && llgauge == gauge && llderiv == deriv;
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  const double2 *u, *m, *ul = nullptr, *lmid = nullptr, *d0;
  double2 *d, *dl = nullptr, *s3, *s5, *t7, *m3;
  if ((rc = smear_in(s, kSmIn0, gauge, mem, &u)) || (rc = smear_in(s, kSmIn1, mid, mem, &m)) ||
      (rc = smear_in(s, kSdIn2, deriv, mem, &d0)))
    return rc;
  d = (double2 *)d0;  // host: the staged copy is updated and copied back
  if (want_long) {
    if ((rc = smear_in(s, kSdIn3, llmid, mem, &lmid))) return rc;
    if (same) {
      ul = u;
      dl = d;
    } else {
      const double2 *dl0;
      if ((rc = smear_in(s, kSmOut0, llgauge, mem, &ul)) || (rc = smear_in(s, kSmOut1, llderiv, mem, &dl0))) return rc;
      dl = (double2 *)dl0;
    }
  }
  if ((rc = smear_scratch(s, *c, &s3, &s5)) || (rc = adj_scratch(s, &t7, &m3))) return rc;
  void *ptmp;
  if ((rc = s->ws.get(kSdTmp, field4_bytes(geo), &ptmp)) ||
      (rc = fat7_dev(geo, *c, u, fs, (double2 *)ptmp, fs, s3, s5)))
    return rc;
  if (same) {
    if ((rc = fat7_adj_dev(geo, *c, u, fs, m, fs, lmid, fs, naik, s3, s5, t7, m3, d, fs, true))) return rc;
  } else {
    if ((rc = fat7_adj_dev(geo, *c, u, fs, m, fs, nullptr, 0, 0.0, s3, s5, t7, m3, d, fs, true))) return rc;
    if (want_long) {
      // the Naik term alone: a level with every fat7 coefficient zero
      qexstag_fat7_coefs z;
      std::memset(&z, 0, sizeof z);
      if ((rc = s->ws.get(kSdTmp, field4_bytes(geo), &ptmp))) return rc;
      QS_CUDA(cudaMemsetAsync(ptmp, 0, field4_bytes(geo), stream()));
      if ((rc = fat7_adj_dev(geo, z, ul, fs, (const double2 *)ptmp, fs, lmid, fs, naik, nullptr, nullptr, t7, m3, dl,
                             fs, true)))
        return rc;
    }
  }
  if ((rc = smear_out_finish(s, d, deriv, mem))) return rc;
  if (want_long && !same && (rc = smear_out_finish(s, dl, llderiv, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_project_u_deriv(qexstag_smear *s, const double *u, const double *x, const double *chain, double *r,
                            double eps, int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!u || !x || !chain || !r) return fail(QEXSTAG_ERR_ARG, "project_u_deriv: null argument");
  const double2 *du, *dx, *dc;
  double2 *dr;
  if ((rc = smear_in(s, kSmIn0, u, mem, &du)) || (rc = smear_in(s, kSmIn1, x, mem, &dx)) ||
      (rc = smear_in(s, kSdIn2, chain, mem, &dc)) || (rc = smear_out_buf(s, kSmOut0, r, mem, &dr)))
    return rc;
  if ((rc = project_u_deriv_dev(s->l->g, du, dx, dc, dr, eps)) || (rc = smear_out_finish(s, dr, r, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_hisq_deriv(qexstag_smear *s, const qexstag_hisq_coefs *c, const double *g, const double *cfat,
                       const double *clong, double *deriv, int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!c || !g || !cfat || !clong || !deriv) return fail(QEXSTAG_ERR_ARG, "hisq_deriv: null argument");
  if (!finite_coefs(c->fat7first) || !finite_coefs(c->fat7second) || !std::isfinite(c->naik))
    return fail(QEXSTAG_ERR_ARG, "hisq_deriv: coefficients not finite");
  const size_t fs = (size_t)9 * s->l->g.V;
  const double2 *u, *cf, *cl;
  double2 *d;
  if ((rc = smear_in(s, kSmIn0, g, mem, &u)) || (rc = smear_in(s, kSmIn1, cfat, mem, &cf)) ||
      (rc = smear_in(s, kSdIn2, clong, mem, &cl)) || (rc = smear_out_buf(s, kSmOut0, deriv, mem, &d)))
    return rc;
  if ((rc = hisq_deriv_dev(s, *c, u, cf, fs, cl, fs, d)) || (rc = smear_out_finish(s, d, deriv, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_hisq_force(qexstag_links *g, qexstag_smear *s, const qexstag_hisq_coefs *c, const double *thin,
                       double *f, const double *phi, double m, const qexstag_solver_params *p,
                       qexstag_solver_stats *st, int mem) {
  int rc;
  if ((rc = check_smear(s, mem))) return rc;
  if (!g || !g->u64 || !c || !thin || !f || !phi || !p) return fail(QEXSTAG_ERR_ARG, "hisq_force: null argument");
  if (g->nl != 8) return fail(QEXSTAG_ERR_ARG, "hisq_force: the link handle must hold 8 (fat+Naik) links");
  if (g->l != s->l) return fail(QEXSTAG_ERR_ARG, "hisq_force: handles on different layouts");
  if (!finite_coefs(c->fat7first) || !finite_coefs(c->fat7second) || !std::isfinite(c->naik))
    return fail(QEXSTAG_ERR_ARG, "hisq_force: coefficients not finite");
  const Geom &geo = s->l->g;
  const size_t fs = (size_t)9 * geo.V;
  const size_t vb = sizeof(double2) * 3 * (size_t)geo.V;
  const double2 *u, *dphi;
  double2 *df;
  void *ppsi, *pf8, *pff;
  if ((rc = smear_in(s, kSmIn0, thin, mem, &u)) || (rc = smear_out_buf(s, kSmOut0, f, mem, &df)) ||
      (rc = s->ws.get(kSfPsi, vb, &ppsi)) || (rc = s->ws.get(kSfF8, 2 * field4_bytes(geo), &pf8)) ||
      (rc = s->ws.get(kSfFF, field4_bytes(geo), &pff)))
    return rc;
  if (mem == QEXSTAG_MEM_DEVICE) {
    dphi = (const double2 *)phi;
  } else {
    void *soa, *aos;
    if ((rc = s->ws.get(kSfPhi, vb, &soa)) || (rc = s->ws.get(kSmAos, field4_bytes(geo) / 4, &aos))) return rc;
    QS_CUDA(cudaMemcpyAsync(aos, phi, vb, cudaMemcpyHostToDevice, stream()));
    if ((rc = aos_to_soa((const double *)aos, (double2 *)soa, geo.V, geo.V, 3))) return rc;
    dphi = (const double2 *)soa;
  }
  // smear the thin links into the operator (smearGetForce's forward part)
  if ((rc = hisq_dev(s, *c, u, g->u64, 2 * fs, g->u64 + fs, 2 * fs))) return rc;
  free_low_links(g->low);
  if ((rc = build_low_links(g))) return rc;
  // stagForceSolve, then fermForce's outer products f1 (fat) and f3 (long)
  double2 *psi = (double2 *)ppsi, *f8 = (double2 *)pf8, *ff = (double2 *)pff;
  const int status = qexstag_force_solve(g, (double *)psi, (const double *)dphi, m, p, st, QEXSTAG_MEM_DEVICE);
  if (status < 0) return status;
  if ((rc = qexstag_ferm_outer(g, (double *)f8, (const double *)psi, QEXSTAG_MEM_DEVICE))) return rc;
  // u.deriv(ff, f1, f3), then projectTAH(ff U^dag)
  if ((rc = hisq_deriv_dev(s, *c, u, f8, 2 * fs, f8 + fs, 2 * fs, ff))) return rc;
  tah_times_adj_kernel<<<field_grid(geo), kSmBlock, 0, stream()>>>(geo.V, ff, u, df, fs);
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = smear_out_finish(s, df, f, mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return status;
}

}  // extern "C"
