/*
 * hmc_oracle.c -- CPU restatement of QEX's gauge action, gauge force and
 * link update.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for qex_b200/csrc/hmcops.cu.
 *
 * Follows (paths relative to the QEX source tree):
 *  - gaugeAction1: S = -(1/nc) (plaq * sum_{x, mu>nu} Re Tr P_munu(x)
 *    + rect * sum_{x, mu!=nu} Re Tr R_munu(x)), R_munu the 2x1 rectangle
 *    with its long side along mu: src/gauge/gaugeAction.nim:487-571;
 *    gaugeActRect / Symanzik coefficients plaq = (1-8 c1) beta,
 *    rect = c1 beta: gaugeAction.nim:51-56.
 *  - gaugeForce = gaugeActionDeriv + contractProjectTAH
 *    (gaugeAction.nim:576-779, src/gauge/gaugeUtils.nim:419-441): with C the
 *    sum of the open paths that close each loop through U_mu(x) (so that
 *    Re Tr[U_mu(x) C] is the loop), F_mu(x) = projectTAH(U_mu(x)
 *    (plaq/nc sum_plaq C + rect/nc sum_rect C)).  Here the paths are formed
 *    directly, one product per loop, rather than through QEX's staple
 *    fields; the sum is the same.
 *  - expAH: scale m by 1/2 until |m|^2 <= 1/16, the degree-12 Taylor
 *    polynomial in m, m^2, m^3, then square back: src/maths/matexp.nim:10-21,
 *    316-346; axexpmuly z = exp(a x) y: src/gauge/gaugeUtils.nim:452-459.
 * Pinned in tests/test_hmc_oracle.py by finite differences of the action
 * against the force, unitarity and group property of expAH, and the
 * free-field action.
 *
 * Layout: gauge fields double[4][V][18] in QEX's V=1 site order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

long or_index(const int L[4], const int x[4]);
void or_coords(const int L[4], int32_t *coord);

typedef struct {
  double r[9], i[9];
} Cm;

static void cm_load(Cm *m, const double *p) {
  for (int e = 0; e < 9; e++) {
    m->r[e] = p[2 * e];
    m->i[e] = p[2 * e + 1];
  }
}
static void cm_store(double *p, const Cm *m) {
  for (int e = 0; e < 9; e++) {
    p[2 * e] = m->r[e];
    p[2 * e + 1] = m->i[e];
  }
}
static Cm cm_mul(const Cm *a, const Cm *b) {
  Cm c;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; k++) {
        re += a->r[3 * i + k] * b->r[3 * k + j] - a->i[3 * i + k] * b->i[3 * k + j];
        im += a->r[3 * i + k] * b->i[3 * k + j] + a->i[3 * i + k] * b->r[3 * k + j];
      }
      c.r[3 * i + j] = re;
      c.i[3 * i + j] = im;
    }
  return c;
}
static Cm cm_dag(const Cm *a) {
  Cm c;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      c.r[3 * i + j] = a->r[3 * j + i];
      c.i[3 * i + j] = -a->i[3 * j + i];
    }
  return c;
}
static void cm_axpy(Cm *y, double a, const Cm *x) {
  for (int e = 0; e < 9; e++) {
    y->r[e] += a * x->r[e];
    y->i[e] += a * x->i[e];
  }
}
static double cm_retr(const Cm *a) { return a->r[0] + a->r[4] + a->r[8]; }

typedef struct {
  int L[4];
  long V;
  int32_t *coord;
  const double *u;
} G;

static long nb(const G *g, long i, const int d[4]) {
  int x[4];
  for (int k = 0; k < 4; k++) x[k] = ((g->coord[4 * i + k] + d[k]) % g->L[k] + g->L[k]) % g->L[k];
  return or_index(g->L, x);
}
/* link of direction mu at site i + d, daggered when dag */
static Cm link(const G *g, long i, int dx0, int dx1, int dx2, int dx3, int mu, int dag) {
  const int d[4] = {dx0, dx1, dx2, dx3};
  Cm m;
  cm_load(&m, g->u + (mu * g->V + nb(g, i, d)) * 18);
  return dag ? cm_dag(&m) : m;
}
#define OFF(mu, a) ((mu) == 0 ? (a) : 0), ((mu) == 1 ? (a) : 0), ((mu) == 2 ? (a) : 0), ((mu) == 3 ? (a) : 0)

/* link at x + a mu + b nu */
static Cm lk(const G *g, long i, int mu, int a, int nu, int b, int dir, int dag) {
  int d[4] = {0, 0, 0, 0};
  d[mu] += a;
  d[nu] += b;
  return link(g, i, d[0], d[1], d[2], d[3], dir, dag);
}

static Cm prod(int n, Cm *m) {
  Cm r = m[0];
  for (int k = 1; k < n; k++) r = cm_mul(&r, &m[k]);
  return r;
}

/* the plaquette and rectangle closers of U_mu(x): open paths from x+mu back
   to x, summed; Re Tr[U_mu(x) C] is the loop */
static void closers(const G *g, long i, int mu, Cm *cp, Cm *cr) {
  memset(cp, 0, sizeof *cp);
  memset(cr, 0, sizeof *cr);
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    for (int s = -1; s <= 1; s += 2) {
      /* hop along s*nu: forward link U_nu(y) or backward U_nu(y - nu)^dag */
#define HOP(a, b, up) (up ? lk(g, i, mu, a, nu, b, nu, 0) : lk(g, i, mu, a, nu, (b) - 1, nu, 1))
#define MUB(a, b) lk(g, i, mu, (a) - 1, nu, b, mu, 1) /* U_mu(x + (a-1) mu + b nu)^dag: step -mu from a */
      const int up = s > 0;
      /* plaquette: x+mu -> x+mu+s nu -> x+s nu -> x */
      Cm p[3] = {HOP(1, 0, up), MUB(1, s), up ? lk(g, i, mu, 0, nu, 0, nu, 1) : lk(g, i, mu, 0, nu, -1, nu, 0)};
      Cm t = prod(3, p);
      cm_axpy(cp, 1.0, &t);
      /* rectangle long in mu, U_mu(x) first: x+mu -> x+2mu -> +s nu -> x+s nu -> x */
      Cm r1[5] = {lk(g, i, mu, 1, nu, 0, mu, 0), HOP(2, 0, up), MUB(2, s), MUB(1, s),
                  up ? lk(g, i, mu, 0, nu, 0, nu, 1) : lk(g, i, mu, 0, nu, -1, nu, 0)};
      t = prod(5, r1);
      cm_axpy(cr, 1.0, &t);
      /* rectangle long in mu, U_mu(x) second: x+mu -> +s nu -> x-mu+s nu -> x-mu -> x */
      Cm r2[5] = {HOP(1, 0, up), MUB(1, s), MUB(0, s),
                  up ? lk(g, i, mu, -1, nu, 0, nu, 1) : lk(g, i, mu, -1, nu, -1, nu, 0), lk(g, i, mu, -1, nu, 0, mu, 0)};
      t = prod(5, r2);
      cm_axpy(cr, 1.0, &t);
      /* rectangle long in nu: x+mu -> x+mu+2s nu -> x+2s nu -> x */
      Cm r3[5] = {HOP(1, 0, up), HOP(1, s, up), MUB(1, 2 * s),
                  up ? lk(g, i, mu, 0, nu, 1, nu, 1) : lk(g, i, mu, 0, nu, -2, nu, 0),
                  up ? lk(g, i, mu, 0, nu, 0, nu, 1) : lk(g, i, mu, 0, nu, -1, nu, 0)};
      t = prod(5, r3);
      cm_axpy(cr, 1.0, &t);
#undef HOP
#undef MUB
    }
  }
}

/* gaugeAction1: each plaquette once (4 links each) and each rectangle once
   (6 links each) */
double or_gauge_action(const int L[4], double plaq, double rect, const double *u) {
  G g = {{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3], NULL, u};
  g.coord = (int32_t *)malloc(sizeof(int32_t) * 4 * g.V);
  or_coords(L, g.coord);
  double sp = 0, sr = 0;
#pragma omp parallel for reduction(+ : sp, sr)
  for (long i = 0; i < g.V; i++)
    for (int mu = 0; mu < 4; mu++) {
      Cm cp, cr;
      closers(&g, i, mu, &cp, &cr);
      Cm um;
      cm_load(&um, u + (mu * g.V + i) * 18);
      Cm a = cm_mul(&um, &cp), b = cm_mul(&um, &cr);
      sp += cm_retr(&a);
      sr += cm_retr(&b);
    }
  free(g.coord);
  return -(plaq * sp / 4.0 + rect * sr / 6.0) / 3.0;
}

static void tah(Cm *r, const Cm *m) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      r->r[3 * i + j] = 0.5 * (m->r[3 * i + j] - m->r[3 * j + i]);
      r->i[3 * i + j] = 0.5 * (m->i[3 * i + j] + m->i[3 * j + i]);
    }
  const double t = (r->i[0] + r->i[4] + r->i[8]) / 3.0;
  r->i[0] -= t;
  r->i[4] -= t;
  r->i[8] -= t;
}

void or_gauge_force(const int L[4], double plaq, double rect, const double *u, double *f) {
  G g = {{L[0], L[1], L[2], L[3]}, (long)L[0] * L[1] * L[2] * L[3], NULL, u};
  g.coord = (int32_t *)malloc(sizeof(int32_t) * 4 * g.V);
  or_coords(L, g.coord);
#pragma omp parallel for
  for (long i = 0; i < g.V; i++)
    for (int mu = 0; mu < 4; mu++) {
      Cm cp, cr, c, um, m, r;
      closers(&g, i, mu, &cp, &cr);
      memset(&c, 0, sizeof c);
      cm_axpy(&c, plaq / 3.0, &cp);
      cm_axpy(&c, rect / 3.0, &cr);
      cm_load(&um, u + (mu * g.V + i) * 18);
      m = cm_mul(&um, &c);
      tah(&r, &m);
      cm_store(f + (mu * g.V + i) * 18, &r);
    }
  free(g.coord);
}

/* expAH (matexp.nim:316-346) */
static Cm exp_ah(const Cm *x) {
  double n2 = 0;
  for (int e = 0; e < 9; e++) n2 += x->r[e] * x->r[e] + x->i[e] * x->i[e];
  double scale = 1.0;
  int ns = 0;
  while (n2 > 1.0 / 16.0) {
    n2 *= 0.25;
    scale *= 0.5;
    ns++;
  }
  Cm m = *x;
  for (int e = 0; e < 9; e++) {
    m.r[e] *= scale;
    m.i[e] *= scale;
  }
  const double C[13] = {1.0, 1.0, 0.5, 1.0 / 6, 1.0 / 24, 1.0 / 120, 1.0 / 720, 1.0 / 5040, 1.0 / 40320,
                        1.0 / 362880, 1.0 / 3628800, 1.0 / 39916800, 1.0 / 479001600};
  Cm m2 = cm_mul(&m, &m), m3 = cm_mul(&m2, &m);
  /* c = C12 m3 + C11 m2 + C10 m + C9; b = c m3 + C8 m2 + C7 m + C6;
     a = b m3 + C5 m2 + C4 m + C3; r = a m3 + C2 m2 + m + 1 */
  Cm c;
  memset(&c, 0, sizeof c);
  cm_axpy(&c, C[12], &m3);
  cm_axpy(&c, C[11], &m2);
  cm_axpy(&c, C[10], &m);
  c.r[0] += C[9];
  c.r[4] += C[9];
  c.r[8] += C[9];
  Cm b = cm_mul(&c, &m3);
  cm_axpy(&b, C[8], &m2);
  cm_axpy(&b, C[7], &m);
  b.r[0] += C[6];
  b.r[4] += C[6];
  b.r[8] += C[6];
  Cm a = cm_mul(&b, &m3);
  cm_axpy(&a, C[5], &m2);
  cm_axpy(&a, C[4], &m);
  a.r[0] += C[3];
  a.r[4] += C[3];
  a.r[8] += C[3];
  Cm r = cm_mul(&a, &m3);
  cm_axpy(&r, C[2], &m2);
  cm_axpy(&r, 1.0, &m);
  r.r[0] += 1.0;
  r.r[4] += 1.0;
  r.r[8] += 1.0;
  for (int k = 0; k < ns; k++) r = cm_mul(&r, &r);
  return r;
}

void or_exp_ah(long n, const double *m, double eps, double *out) {
#pragma omp parallel for
  for (long k = 0; k < n; k++) {
    Cm x;
    cm_load(&x, m + 18 * k);
    for (int e = 0; e < 9; e++) {
      x.r[e] *= eps;
      x.i[e] *= eps;
    }
    Cm r = exp_ah(&x);
    cm_store(out + 18 * k, &r);
  }
}

/* axexpmuly(u, eps, p, u): u = expAH(eps p) u per link */
void or_link_update(long n, double *u, const double *p, double eps) {
#pragma omp parallel for
  for (long k = 0; k < n; k++) {
    Cm x, y;
    cm_load(&x, p + 18 * k);
    cm_load(&y, u + 18 * k);
    for (int e = 0; e < 9; e++) {
      x.r[e] *= eps;
      x.i[e] *= eps;
    }
    Cm r = exp_ah(&x);
    Cm z = cm_mul(&r, &y);
    cm_store(u + 18 * k, &z);
  }
}
