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
