/*
 * smear_oracle.c -- CPU restatement of QEX's HISQ link smearing.
 *
 * TEST INFRASTRUCTURE ONLY.  The checker for the library's smearing kernels
 * (qex_b200/csrc/smear.cu); the product path never calls it.
 *
 * PARITY UNPINNED, as for qexstag_oracle.c: QEX (Nim) cannot be built here
 * and stores no smeared-link vectors.  This restatement is pinned in
 * tests/test_smear_oracle.py by known answers: phased unit links smear to
 * (c1 + 6 cL - 6 c3 + 24 c5 - 48 c7) times the phases (9/8 for HISQ's second
 * level, 1 for its first), gauge covariance of fat7, projectU and the whole
 * HISQ smearing, and projectU giving a unitary matrix that equals
 * X (X^dagger X)^(-1/2) computed by an independent eigen-decomposition.
 *
 * Follows (paths relative to the QEX source tree):
 *  - computeGenStaple:           src/gauge/fat7l.nim:24-68
 *  - makeImpLinks (fat7 + Naik): src/gauge/fat7l.nim:70-154
 *  - setHisqFat7 / HisqCoefs.init: src/physics/hisqLinks.nim:10-27
 *  - HisqCoefs.smear:            src/physics/hisqLinks.nim:40-46
 *  - newHISQ:                    src/gauge/hisqsmear.nim:53-64
 *  - projectU (Cayley-Hamilton): src/maths/matrixFunctions.nim:118-150,
 *                                165-212, 340-351
 *  - symStaple / symStapleDeriv: src/gauge/smearutil.nim:3-56
 *  - fat7lDeriv (with Naik):     src/gauge/fat7lderiv.nim:122-331
 *  - projectUderiv, sylsolve:    src/maths/matrixFunctions.nim:360-390,
 *                                src/maths/projUderiv.nim:96-145
 *  - smearGetForce's chain rule: src/gauge/hisqsmear.nim:66-105
 * The chain rule is pinned by QEX's own check (hisqsmear.nim:126-168):
 * finite differences of sum Re Tr (C^dag fat + Cl^dag long) along random
 * directions, for one-link-only, fat7-only and full HISQ coefficients.
 *
 * Layout: a gauge field is double[4][V][3][3][2] (direction, QEX V=1 site
 * index, row-major 3x3, re/im); coefficient arrays are
 * {oneLink, threeStaple, fiveStaple, sevenStaple, lepage}.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

long or_index(const int L[4], const int x[4]);
void or_coords(const int L[4], int32_t *coord);

typedef struct {
  int L[4];
  long V;
  int32_t *coord;
} SGeo;

static void sgeo_init(SGeo *s, const int L[4]) {
  for (int d = 0; d < 4; d++) s->L[d] = L[d];
  s->V = (long)L[0] * L[1] * L[2] * L[3];
  s->coord = (int32_t *)malloc(sizeof(int32_t) * 4 * s->V);
  or_coords(L, s->coord);
}

/* out(x) = in(x + len*mu): QEX's Shifter `^*` (forward shift) */
static void shift_m(const SGeo *s, double *out, const double *in, int mu, int len) {
#pragma omp parallel for
  for (long i = 0; i < s->V; i++) {
    int x[4] = {s->coord[4 * i], s->coord[4 * i + 1], s->coord[4 * i + 2], s->coord[4 * i + 3]};
    x[mu] = ((x[mu] + len) % s->L[mu] + s->L[mu]) % s->L[mu];
    memcpy(out + 18 * i, in + 18 * or_index(s->L, x), 18 * sizeof(double));
  }
}

/* 3x3 complex products: r = a b, a b^dagger, a^dagger b (r not aliased) */
static void m_nn(double *r, const double *a, const double *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        const double *p = a + 2 * (3 * i + k), *q = b + 2 * (3 * k + j);
        re += p[0] * q[0] - p[1] * q[1];
        im += p[0] * q[1] + p[1] * q[0];
      }
      r[2 * (3 * i + j)] = re;
      r[2 * (3 * i + j) + 1] = im;
    }
}
static void m_nd(double *r, const double *a, const double *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        const double *p = a + 2 * (3 * i + k), *q = b + 2 * (3 * j + k);
        re += p[0] * q[0] + p[1] * q[1];
        im += p[1] * q[0] - p[0] * q[1];
      }
      r[2 * (3 * i + j)] = re;
      r[2 * (3 * i + j) + 1] = im;
    }
}
static void m_dn(double *r, const double *a, const double *b) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        const double *p = a + 2 * (3 * k + i), *q = b + 2 * (3 * k + j);
        re += p[0] * q[0] + p[1] * q[1];
        im += p[0] * q[1] - p[1] * q[0];
      }
      r[2 * (3 * i + j)] = re;
      r[2 * (3 * i + j) + 1] = im;
    }
}

/* field ops over V sites */
static void f_nn(const SGeo *s, double *r, const double *a, const double *b) {
#pragma omp parallel for
  for (long i = 0; i < s->V; i++) m_nn(r + 18 * i, a + 18 * i, b + 18 * i);
}
static void f_nd(const SGeo *s, double *r, const double *a, const double *b) {
#pragma omp parallel for
  for (long i = 0; i < s->V; i++) m_nd(r + 18 * i, a + 18 * i, b + 18 * i);
}
static void f_dn(const SGeo *s, double *r, const double *a, const double *b) {
#pragma omp parallel for
  for (long i = 0; i < s->V; i++) m_dn(r + 18 * i, a + 18 * i, b + 18 * i);
}
static void f_axpy(const SGeo *s, double *y, double a, const double *x) {
#pragma omp parallel for
  for (long i = 0; i < 18 * s->V; i++) y[i] += a * x[i];
}

/* fat7l.nim:24-68.  gauge[nu] * (link shifted by +nu) * (gauge[nu] shifted by
   +mu)^dagger plus the same path hung below: (gauge[nu]^dagger link
   gauge[nu](x+mu)) shifted by -nu.  With staple != NULL the sum is stored and
   added to fl with weight coef; otherwise the two halves are added to fl one
   after the other. */
static void gen_staple(const SGeo *s, double *staple, int mu, int nu, const double *link, double coef,
                       const double *const gauge[4], double *fl, double *w) {
  const long n = 18 * s->V;
  double *ts0 = w, *ts1 = w + n, *t = w + 2 * n, *ts2 = w + 3 * n;
  shift_m(s, ts0, link, nu, 1);          /* link(x+nu) */
  shift_m(s, ts1, gauge[nu], mu, 1);     /* U_nu(x+mu) */
  f_nn(s, t, gauge[nu], ts0);
  if (staple) {
    f_nd(s, staple, t, ts1);
  } else {
    f_nd(s, ts0, t, ts1);
    f_axpy(s, fl, coef, ts0);
  }
  f_dn(s, t, gauge[nu], link);           /* U_nu^dagger link U_nu(x+mu) */
  f_nn(s, ts0, t, ts1);
  shift_m(s, ts2, ts0, nu, -1);
  if (staple) {
    f_axpy(s, staple, 1.0, ts2);
    f_axpy(s, fl, coef, staple);
  } else {
    f_axpy(s, fl, coef, ts2);
  }
}

/* makeImpLinks (fat7l.nim:70-154).  gf, fl: [4][V][18]; gfl, ll may be NULL
   (no long links) */
void or_fat7(const int L[4], const double *coef, const double *gf, double *fl, const double *gfl,
             double *ll, double naik) {
  SGeo s;
  sgeo_init(&s, L);
  const long n = 18 * s.V;
  double coef1 = coef[0], coef3 = coef[1], coef5 = coef[2], coef7 = coef[3], coefL = coef[4];
  const int have5 = (coef5 != 0.0) || (coef7 != 0.0) || (coefL != 0.0);
  const int have3 = (coef3 != 0.0) || have5;
  coef1 -= 6.0 * coefL;  /* the Lepage term below includes 6 one-link paths */
  const double *g[4] = {gf, gf + n, gf + 2 * n, gf + 3 * n};
  double *staple = (double *)malloc(sizeof(double) * n);
  double *tmp1 = (double *)malloc(sizeof(double) * n);
  double *w = (double *)malloc(sizeof(double) * 4 * n);
  for (int dir = 0; dir < 4; dir++) {
    double *f = fl + dir * n;
    for (long i = 0; i < n; i++) f[i] = coef1 * g[dir][i];
    if (!have3) continue;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == dir) continue;
      gen_staple(&s, staple, dir, nu, g[dir], coef3, g, f, w);
      if (coefL != 0.0) gen_staple(&s, NULL, dir, nu, staple, coefL, g, f, w);
      if (coef5 != 0.0 || coef7 != 0.0) {
        for (int rho = 0; rho < 4; rho++) {
          if (rho == dir || rho == nu) continue;
          gen_staple(&s, tmp1, dir, rho, staple, coef5, g, f, w);
          if (coef7 != 0.0)
            for (int sig = 0; sig < 4; sig++)
              if (sig != dir && sig != nu && sig != rho) gen_staple(&s, NULL, dir, sig, tmp1, coef7, g, f, w);
        }
      }
    }
  }
  if (naik != 0.0 && gfl && ll) {
    for (int dir = 0; dir < 4; dir++) {
      const double *u = gfl + dir * n;
      shift_m(&s, w, u, dir, 1);        /* U(x+mu) */
      f_nn(&s, w + n, u, w);            /* U(x) U(x+mu) */
      shift_m(&s, w + 2 * n, w + n, dir, 1);
      f_nn(&s, ll + dir * n, u, w + 2 * n);
      for (long i = 0; i < n; i++) ll[dir * n + i] *= naik;
    }
  }
  free(staple);
  free(tmp1);
  free(w);
  free(s.coord);
}

/* eigenvalues of a Hermitian 3x3 matrix from tr, tr(t^2), det
   (matrixFunctions.nim:118-150, trigonometric solution of the cubic) */
static void eigs3(double *e0, double *e1, double *e2, double tr, double p2, double det) {
  const double tr3 = tr / 3.0, p23 = p2 / 3.0, tr32 = tr3 * tr3;
  const double q = fabs(0.5 * (p23 - tr32));
  const double r = 0.25 * tr3 * (5.0 * tr32 - p2) - 0.5 * det;
  const double sq = sqrt(q), sq3 = q * sq;
  double isq3 = 1.0 / sq3;
  if (isq3 > 3e38) isq3 = 3e38;
  if (isq3 < -3e38) isq3 = -3e38;
  double rsq3 = r * isq3;
  if (rsq3 > 1.0) rsq3 = 1.0;
  if (rsq3 < -1.0) rsq3 = -1.0;
  const double t = acos(rsq3) / 3.0;
  const double sqc = sq * cos(t), sqs = 1.73205080756887729352 * sq * sin(t);
  *e0 = tr3 - 2.0 * sqc;
  *e1 = tr3 + sqc + sqs;
  *e2 = tr3 + sqc - sqs;
}

/* r = x (x^dagger x + eps)^(-1/2) (matrixFunctions.nim:340-351 with the
   Cayley-Hamilton inverse square root of 165-212) */
static void project_u1(double *r, const double *x, double eps) {
  double t[18], t2[18], z[18];
  m_dn(t, x, x);
  t[0] += eps;
  t[8] += eps;
  t[16] += eps;
  m_nn(t2, t, t);
  const double tr = t[0] + t[8] + t[16];
  const double p2 = t2[0] + t2[8] + t2[16];
  /* Re det t */
  double c[18];
  memcpy(c, t, sizeof c);
#define RE(m, i, j) m[2 * (3 * (i) + (j))]
#define IM(m, i, j) m[2 * (3 * (i) + (j)) + 1]
  double m00r = RE(c, 1, 1) * RE(c, 2, 2) - IM(c, 1, 1) * IM(c, 2, 2) - (RE(c, 1, 2) * RE(c, 2, 1) - IM(c, 1, 2) * IM(c, 2, 1));
  double m00i = RE(c, 1, 1) * IM(c, 2, 2) + IM(c, 1, 1) * RE(c, 2, 2) - (RE(c, 1, 2) * IM(c, 2, 1) + IM(c, 1, 2) * RE(c, 2, 1));
  double m01r = RE(c, 1, 2) * RE(c, 2, 0) - IM(c, 1, 2) * IM(c, 2, 0) - (RE(c, 1, 0) * RE(c, 2, 2) - IM(c, 1, 0) * IM(c, 2, 2));
  double m01i = RE(c, 1, 2) * IM(c, 2, 0) + IM(c, 1, 2) * RE(c, 2, 0) - (RE(c, 1, 0) * IM(c, 2, 2) + IM(c, 1, 0) * RE(c, 2, 2));
  double m02r = RE(c, 1, 0) * RE(c, 2, 1) - IM(c, 1, 0) * IM(c, 2, 1) - (RE(c, 1, 1) * RE(c, 2, 0) - IM(c, 1, 1) * IM(c, 2, 0));
  double m02i = RE(c, 1, 0) * IM(c, 2, 1) + IM(c, 1, 0) * RE(c, 2, 1) - (RE(c, 1, 1) * IM(c, 2, 0) + IM(c, 1, 1) * RE(c, 2, 0));
  const double det = RE(c, 0, 0) * m00r - IM(c, 0, 0) * m00i + RE(c, 0, 1) * m01r - IM(c, 0, 1) * m01i +
                     RE(c, 0, 2) * m02r - IM(c, 0, 2) * m02i;
#undef RE
#undef IM
  double l0, l1, l2;
  eigs3(&l0, &l1, &l2, tr, p2, det);
  const double s0 = sqrt(fabs(l0)), s1 = sqrt(fabs(l1)), s2 = sqrt(fabs(l2));
  const double u = s0 + s1 + s2, w = s0 * s1 * s2;
  const double d = w * (s0 + s1) * (s0 + s2) * (s1 + s2);
  const double di = 1.0 / d;
  const double c0 = (w * u * u + l0 * s0 * (l1 + l2) + l1 * s1 * (l0 + l2) + l2 * s2 * (l0 + l1)) * di;
  const double c1 = -(tr * u + w) * di;
  const double c2 = u * di;
  for (int i = 0; i < 18; i++) z[i] = c1 * t[i] + c2 * t2[i];
  z[0] += c0;
  z[8] += c0;
  z[16] += c0;
  m_nn(r, x, z);
}

/* projectU of n matrices */
void or_project_u(long n, const double *x, double *r, double eps) {
#pragma omp parallel for
  for (long i = 0; i < n; i++) project_u1(r + 18 * i, x + 18 * i, eps);
}

/* HisqCoefs.smear (hisqLinks.nim:40-46): t1 = fat7(g, first); t2 =
   projectU(t1); fl = fat7(t2, second), ll = naik * t2 t2 t2 */
void or_hisq_smear(const int L[4], const double *first, const double *second, double naik, double eps,
                   const double *g, double *fl, double *ll) {
  const long V = (long)L[0] * L[1] * L[2] * L[3];
  const long n = 4 * 18 * V;
  double *t1 = (double *)malloc(sizeof(double) * n);
  double *t2 = (double *)malloc(sizeof(double) * n);
  or_fat7(L, first, g, t1, NULL, NULL, 0.0);
  or_project_u(4 * V, t1, t2, eps);
  or_fat7(L, second, t2, fl, t2, ll, naik);
  free(t1);
  free(t2);
}

/* ------------------------------------------------------------------ */
/* chain rule through the smearing                                     */
/* ------------------------------------------------------------------ */
/* Convention (QEX's, src/gauge/hisqsmear.nim:111-168): for a chain C on an
   output field and S = sum_x Re Tr C(x)^dagger out(x), the derivative with
   respect to an input field U is the field f with dS = sum Re Tr dU^dagger f. */

static void m_dd(double *r, const double *a, const double *b) { /* a^dag b^dag */
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        const double *p = a + 2 * (3 * k + i), *q = b + 2 * (3 * j + k);
        re += p[0] * q[0] - p[1] * q[1];
        im += -p[0] * q[1] - p[1] * q[0];
      }
      r[2 * (3 * i + j)] = re;
      r[2 * (3 * i + j) + 1] = im;
    }
}
static void f_dd(const SGeo *s, double *r, const double *a, const double *b) {
#pragma omp parallel for
  for (long i = 0; i < s->V; i++) m_dd(r + 18 * i, a + 18 * i, b + 18 * i);
}

/* symStaple (src/gauge/smearutil.nim:3-20): s += alp [g1 g2(x+d1) g1(x+d2)^dag
   + (g1^dag g2 g1(x+d2))(x-d1)], g1 the side field of direction d1, g2 the
   middle field of direction d2 */
static void sym_staple(const SGeo *s, double *st, double alp, const double *g1, const double *g2, int d1, int d2,
                       double *w) {
  const long n = 18 * s->V;
  double *s1 = w, *s2 = w + n, *t = w + 2 * n, *tm = w + 3 * n, *sm = w + 4 * n;
  shift_m(s, s1, g1, d2, 1);
  shift_m(s, s2, g2, d1, 1);
  f_dn(s, t, g1, g2);
  f_nn(s, tm, t, s1);
  shift_m(s, sm, tm, d1, -1);
  f_nn(s, t, g1, s2);
  f_nd(s, tm, t, s1);
  f_axpy(s, st, alp, tm);
  f_axpy(s, st, alp, sm);
}

/* symStapleDeriv (src/gauge/smearutil.nim:22-56): with chain c on
   symStaple(g1, g2), f1 += derivative w.r.t. g1 and f2 += derivative w.r.t.
   g2 */
static void sym_staple_deriv(const SGeo *s, double *f1, double *f2, const double *g1, const double *g2, int d1,
                             int d2, const double *c, double *w) {
  const long n = 18 * s->V;
  double *s1 = w, *s2 = w + n, *sc = w + 2 * n, *t = w + 3 * n, *tm1 = w + 4 * n, *tm2 = w + 5 * n,
         *sm = w + 6 * n, *u = w + 7 * n;
  shift_m(s, s1, g1, d2, 1);
  shift_m(s, s2, g2, d1, 1);
  shift_m(s, sc, c, d1, 1);
  f_dn(s, t, g1, c);
  f_nn(s, tm1, t, s1);      /* g1^dag c s1 */
  f_dn(s, t, g2, g1);
  f_nn(s, tm2, t, sc);      /* g2^dag g1 s */
  f_dn(s, t, c, g1);
  f_nn(s, u, t, s2);        /* c^dag g1 s2 */
  f_axpy(s, tm2, 1.0, u);
  f_nn(s, t, g2, s1);
  f_nd(s, u, t, sc);
  f_axpy(s, f1, 1.0, u);    /* g2 s1 s^dag */
  f_nn(s, t, c, s1);
  f_nd(s, u, t, s2);
  f_axpy(s, f1, 1.0, u);    /* c s1 s2^dag */
  f_nn(s, t, g1, sc);
  f_nd(s, u, t, s1);
  f_axpy(s, f2, 1.0, u);    /* g1 s s1^dag */
  shift_m(s, sm, tm1, d1, -1);
  f_axpy(s, f2, 1.0, sm);
  shift_m(s, sm, tm2, d2, -1);
  f_axpy(s, f1, 1.0, sm);
}

/* fat7lDeriv (src/gauge/fat7lderiv.nim:122-331): deriv += d/d gauge of
   sum Re Tr mid^dag fat7(gauge); when naik != 0 and ll fields are given,
   llderiv += d/d llgauge of sum Re Tr llmid^dag naik U(x)U(x+mu)U(x+2mu).
   All fields [4][V][18]. */
void or_fat7_deriv(const int L[4], const double *coef, const double *gauge, const double *mid, double *deriv,
                   const double *llgauge, const double *llmid, double *llderiv, double naik) {
  SGeo s;
  sgeo_init(&s, L);
  const long n = 18 * s.V;
  const double coefL = coef[4], coef1 = coef[0] - 6.0 * coefL, coef3 = coef[1], coef5 = coef[2], coef7 = coef[3];
  const int have5 = (coef5 != 0.0) || (coef7 != 0.0) || (coefL != 0.0);
  const int have3 = (coef3 != 0.0) || have5;
  const double *g[4], *md[4];
  double *dv[4];
  for (int d = 0; d < 4; d++) {
    g[d] = gauge + d * n;
    md[d] = mid + d * n;
    dv[d] = deriv + d * n;
  }
  double *stpl3 = (double *)calloc(4 * n, sizeof(double));
  double *mid5 = (double *)calloc(4 * n, sizeof(double));
  double *stpl5 = (double *)malloc(sizeof(double) * n);
  double *mid3 = (double *)malloc(sizeof(double) * n);
  double *w = (double *)malloc(sizeof(double) * 8 * n);
  for (int sig = 0; sig < 4; sig++) {
    if (have5) {
      for (int mu = 0; mu < 4; mu++) {
        if (mu == sig) continue;
        memset(stpl3 + mu * n, 0, sizeof(double) * n);
        sym_staple(&s, stpl3 + mu * n, 1.0, g[mu], g[sig], mu, sig, w);
        memset(mid5 + mu * n, 0, sizeof(double) * n);
      }
      for (int rho = 0; rho < 4; rho++) {
        if (rho == sig) continue;
        memset(stpl5, 0, sizeof(double) * n);
        if (coef7 != 0.0) {
          for (int mu = 0; mu < 4; mu++) {
            if (mu == sig || mu == rho) continue;
            for (int nu = 0; nu < 4; nu++) {
              if (nu == sig || nu == rho || nu == mu) continue;
              sym_staple(&s, stpl5, 1.0, g[nu], stpl3 + mu * n, nu, sig, w);
            }
          }
          for (long i = 0; i < n; i++) stpl5[i] *= coef7;
        }
        memset(mid3, 0, sizeof(double) * n);
        if (coefL != 0.0) f_axpy(&s, stpl5, coefL, stpl3 + rho * n);
        if (coefL != 0.0 || coef7 != 0.0) sym_staple_deriv(&s, dv[rho], mid3, g[rho], stpl5, rho, sig, md[sig], w);
        if (coefL != 0.0) f_axpy(&s, mid5 + rho * n, coefL, mid3);
        for (long i = 0; i < n; i++) mid3[i] *= coef7;
        f_axpy(&s, mid3, coef5, md[sig]);
        for (int mu = 0; mu < 4; mu++) {
          if (mu == sig || mu == rho) continue;
          for (int nu = 0; nu < 4; nu++) {
            if (nu == sig || nu == rho || nu == mu) continue;
            sym_staple_deriv(&s, dv[mu], mid5 + nu * n, g[mu], stpl3 + nu * n, mu, sig, mid3, w);
          }
        }
      }
    }
    if (have3) {
      memset(mid3, 0, sizeof(double) * n);
      for (int mu = 0; mu < 4; mu++) {
        if (mu == sig) continue;
        for (long i = 0; i < n; i++) stpl5[i] = coef3 * md[sig][i] + (have5 ? mid5[mu * n + i] : 0.0);
        sym_staple_deriv(&s, dv[mu], mid3, g[mu], g[sig], mu, sig, stpl5, w);
      }
      f_axpy(&s, dv[sig], 1.0, mid3);
    }
    if (coef1 != 0.0) f_axpy(&s, dv[sig], coef1, md[sig]);
  }
  if (naik != 0.0 && llgauge && llmid && llderiv) {
    double *sa = w, *tm1 = w + n, *sm = w + 2 * n, *tm2 = w + 3 * n, *sb = w + 4 * n, *t = w + 5 * n;
    for (int mu = 0; mu < 4; mu++) {
      const double *lg = llgauge + mu * n, *lm = llmid + mu * n;
      double *ld = llderiv + mu * n;
      shift_m(&s, sa, lg, mu, 1);          /* U(x+mu) */
      f_dn(&s, tm1, lg, lm);               /* U^dag mid */
      shift_m(&s, sm, tm1, mu, -1);
      f_dd(&s, tm2, sa, lg);               /* U(x+mu)^dag U^dag */
      shift_m(&s, sb, tm2, mu, 1);
      f_nd(&s, t, sm, sa);
      f_axpy(&s, ld, naik, t);
      f_dn(&s, tm1, lg, sm);
      shift_m(&s, sm, tm1, mu, -1);
      f_nn(&s, t, lm, sb);
      f_axpy(&s, t, 1.0, sm);
      f_axpy(&s, ld, naik, t);
    }
  }
  free(stpl3);
  free(mid5);
  free(stpl5);
  free(mid3);
  free(w);
  free(s.coord);
}

/* 3x3 inverse through the adjugate */
static void m_adjugate(double *r, const double *x) {
#define XR(i, j) x[2 * (3 * (i) + (j))]
#define XI(i, j) x[2 * (3 * (i) + (j)) + 1]
  /* r_ij = x_ab x_cd - x_ef x_gh with the index pattern of the cofactors */
  static const int P[9][8] = {{1, 1, 2, 2, 1, 2, 2, 1}, {2, 1, 0, 2, 2, 2, 0, 1}, {0, 1, 1, 2, 0, 2, 1, 1},
                              {1, 2, 2, 0, 1, 0, 2, 2}, {2, 2, 0, 0, 2, 0, 0, 2}, {0, 2, 1, 0, 0, 0, 1, 2},
                              {1, 0, 2, 1, 1, 1, 2, 0}, {2, 0, 0, 1, 2, 1, 0, 0}, {0, 0, 1, 1, 0, 1, 1, 0}};
  for (int e = 0; e < 9; e++) {
    const int *p = P[e];
    const double ar = XR(p[0], p[1]), ai = XI(p[0], p[1]), br = XR(p[2], p[3]), bi = XI(p[2], p[3]);
    const double cr = XR(p[4], p[5]), ci = XI(p[4], p[5]), dr = XR(p[6], p[7]), di = XI(p[6], p[7]);
    r[2 * e] = (ar * br - ai * bi) - (cr * dr - ci * di);
    r[2 * e + 1] = (ar * bi + ai * br) - (cr * di + ci * dr);
  }
#undef XR
#undef XI
}

static void m_inverse(double *r, const double *x) {
  double ad[18];
  m_adjugate(ad, x);
  /* det = sum_k x_0k ad_k0 */
  double dr = 0, di = 0;
  for (int k = 0; k < 3; k++) {
    const double *a = x + 2 * k, *b = ad + 2 * (3 * k);
    dr += a[0] * b[0] - a[1] * b[1];
    di += a[0] * b[1] + a[1] * b[0];
  }
  const double nn = dr * dr + di * di, ir = dr / nn, ii = -di / nn;
  for (int e = 0; e < 9; e++) {
    const double a = ad[2 * e], b = ad[2 * e + 1];
    r[2 * e] = a * ir - b * ii;
    r[2 * e + 1] = a * ii + b * ir;
  }
}

/* sylsolve (src/maths/projUderiv.nim:96-145, 3x3 branch): x with
   a x + x a = c, from the adjugate of a and its invariants (a Hermitian
   positive here, so the invariants are taken real) */
static void sylsolve3(double *x, const double *a, const double *c) {
  double ad[18], ac[18], ca[18], aca[18], adc[18], cad[18], adcad[18];
  m_adjugate(ad, a);
  const double t = a[0] + a[8] + a[16];
  const double s = ad[0] + ad[8] + ad[16];
  double r = 0;
  for (int k = 0; k < 3; k++) r += a[2 * k] * ad[2 * (3 * k)] - a[2 * k + 1] * ad[2 * (3 * k) + 1];
  m_nn(ac, a, c);
  m_nn(ca, c, a);
  m_nn(aca, ac, a);
  m_nn(adc, ad, c);
  m_nn(cad, c, ad);
  m_nn(adcad, adc, ad);
  const double c2 = 1.0 / (2.0 * (s * t - r));
  const double c0 = c2 * (s + t * t), c1 = c2 * (t / r), c4 = c2 * t;
  for (int i = 0; i < 18; i++)
    x[i] = c0 * c[i] + c1 * adcad[i] + c2 * (aca[i] - adc[i] - cad[i]) - c4 * (ac[i] + ca[i]);
}

/* inverse square root of x^dagger x + eps (projectUrsqrt,
   matrixFunctions.nim:340-346) */
static void rsqrt_xdx(double *z, const double *x, double eps) {
  /* projectU computes x z; recover z = x^-1 (x z) would lose accuracy, so
     repeat its inner steps */
  double t[18], t2[18];
  m_dn(t, x, x);
  t[0] += eps;
  t[8] += eps;
  t[16] += eps;
  m_nn(t2, t, t);
  const double tr = t[0] + t[8] + t[16];
  const double p2 = t2[0] + t2[8] + t2[16];
  double ad[18];
  m_adjugate(ad, t);
  double det = 0;
  for (int k = 0; k < 3; k++) det += t[2 * k] * ad[2 * (3 * k)] - t[2 * k + 1] * ad[2 * (3 * k) + 1];
  double l0, l1, l2;
  eigs3(&l0, &l1, &l2, tr, p2, det);
  const double s0 = sqrt(fabs(l0)), s1 = sqrt(fabs(l1)), s2 = sqrt(fabs(l2));
  const double u = s0 + s1 + s2, w = s0 * s1 * s2;
  const double di = 1.0 / (w * (s0 + s1) * (s0 + s2) * (s1 + s2));
  const double c0 = (w * u * u + l0 * s0 * (l1 + l2) + l1 * s1 * (l0 + l2) + l2 * s2 * (l0 + l1)) * di;
  const double c1 = -(tr * u + w) * di, c2 = u * di;
  for (int i = 0; i < 18; i++) z[i] = c1 * t[i] + c2 * t2[i];
  z[0] += c0;
  z[8] += c0;
  z[16] += c0;
}

/* projectUderiv (matrixFunctions.nim:368-390): r = d/dx of
   Re Tr chain^dagger projectU(x), with u = projectU(x).  r may alias chain. */
static void project_u_deriv1(double *r, const double *u, const double *x, const double *chain, double eps) {
  double z[18], y[18], t1[18], t2[18], cz[18];
  rsqrt_xdx(z, x, eps);
  m_inverse(y, z);
  m_nn(cz, chain, z);
  m_dn(t1, u, cz);
  sylsolve3(t2, y, t1);
  for (int i = 0; i < 9; i++) {  /* t1 = t2 + t2^dagger */
    const int p = i / 3, q = i % 3, e = 3 * q + p;
    t1[2 * i] = t2[2 * i] + t2[2 * e];
    t1[2 * i + 1] = t2[2 * i + 1] - t2[2 * e + 1];
  }
  m_nn(t2, x, t1);
  for (int i = 0; i < 18; i++) r[i] = cz[i] - t2[i];
}

void or_project_u_deriv(long n, const double *u, const double *x, const double *chain, double *r, double eps) {
#pragma omp parallel for
  for (long i = 0; i < n; i++) project_u_deriv1(r + 18 * i, u + 18 * i, x + 18 * i, chain + 18 * i, eps);
}

void or_sylsolve(long n, const double *a, const double *c, double *x) {
  for (long i = 0; i < n; i++) sylsolve3(x + 18 * i, a + 18 * i, c + 18 * i);
}

/* the chain rule of HisqCoefs' smearing (smearGetForce's smearedForce,
   src/gauge/hisqsmear.nim:66-105): deriv = d/dg of
   sum Re Tr (cfat^dag fat(g) + clong^dag long(g)) */
void or_hisq_deriv(const int L[4], const double *first, const double *second, double naik, double eps,
                   const double *g, const double *cfat, const double *clong, double *deriv) {
  const long V = (long)L[0] * L[1] * L[2] * L[3];
  const long n = 4 * 18 * V;
  double *v = (double *)malloc(sizeof(double) * n);
  double *w = (double *)malloc(sizeof(double) * n);
  double *f = (double *)calloc(n, sizeof(double));
  double *fll = (double *)calloc(n, sizeof(double));
  or_fat7(L, first, g, v, NULL, NULL, 0.0);
  or_project_u(4 * V, v, w, eps);
  or_fat7_deriv(L, second, w, cfat, f, w, clong, fll, naik);
  for (long i = 0; i < n; i++) f[i] += fll[i];
  or_project_u_deriv(4 * V, w, v, f, f, eps);
  memset(deriv, 0, sizeof(double) * n);
  or_fat7_deriv(L, first, g, f, deriv, NULL, NULL, NULL, 0.0);
  free(v);
  free(w);
  free(f);
  free(fll);
}
