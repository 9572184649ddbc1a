/*
 * qexstag_oracle.c -- CPU restatement of QEX's staggered-fermion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
 * (qex_b200/csrc): tests, the smoke check and the CPU-baseline leg of the
 * benchmark may call it; the product path never does.
 *
 * PARITY PINNED AT THE SOLVER LEVEL, NOT ELEMENT BY ELEMENT.  QEX is written
 * in Nim and no Nim compiler exists on the build or GPU machines, so QEX's
 * own stagD/CG cannot be run to produce reference outputs, and QEX stores no
 * golden vectors at the Dslash / CG / force level.  Its HISQ HMC regression
 * logs (src/alphas/regression/) do record the first solves of a cold-start
 * 8^3 x 16 trajectory: with the HISQ smearing of phased unit links, D and the
 * full-lattice solve restated here, this oracle takes the same iteration
 * counts (26, 26, 34) and ends at residuals of the same size
 * (tests/test_oracle_qex_regression.py, fixture tests/golden/).  Element by
 * element the restatement is pinned by analytic known answers, checked in
 * tests/test_oracle.py: the free-field spectrum 4(m^2 + sum_mu sin^2 p_mu)
 * with antiperiodic time, antihermiticity of the hopping term, gauge
 * covariance, the Schur identity, CG/multi-shift residuals and central finite
 * differences of the action against the force.
 *
 * Conventions restated from QEX (paths relative to the QEX source tree):
 *  - site index, V=1 layout, one rank: src/layout/qlayout.nim:108-136
 *    lex = x0 + L0(x1 + L1(x2 + L2 x3)); idx = (lex + (sum x odd ? V : 0))/2
 *  - shift tables: src/layout/qshifts.nim:187-223, src/layout/shiftX.nim:76-101
 *    pidx[i] = index of x(i) + len*mu (periodic)
 *  - staggered phases [8,9,11,0]: src/physics/stagD.nim:560-571
 *  - antiperiodic time boundary (setBC): src/gauge/gaugeUtils.nim:133-140
 *  - stagD2: src/physics/stagD.nim:383-448
 *  - stagD / D / Ddag: src/physics/stagD.nim:459-462, 617-622
 *  - stagD2ee (stagDP then stagDM): src/physics/stagD.nim:485-512
 *  - eoReconstruct: src/physics/stagD.nim:633-637
 *  - CG (cpNone): src/solvers/cg.nim:55-272
 *  - solveXX defect correction: src/physics/stagSolve.nim:330-421
 *  - solve / solveInner / solveReconL / solveReconR:
 *    src/physics/stagSolve.nim:238-326, 469-557
 *  - multi-shift CG: src/solvers/cgm.nim:68-246; driver
 *    src/physics/stagSolve.nim:560-668
 *  - force solve + fermForce (no smearing): src/hmc/hmcAction.nim:669-790
 *  - projectTAH: src/maths/matrixFunctions.nim:414-419
 *
 * Data layout used by every entry point (the QEX V=1 layout):
 *  - colour vector field: double[V][3][2]   (site index, colour, re/im)
 *  - link field list:     double[nlinks][V][3][3][2]  (row-major 3x3)
 *    nlinks == 4: naive, link k is direction k with hop +1;
 *    nlinks == 8: fat+Naik interleaved as QEX's newStag3 does
 *    (stagD.nim:40-51, 603-615): k = 2*mu is the one-hop fat link,
 *    k = 2*mu+1 the three-hop long link.
 *  Links are expected with staggered phases and boundary signs folded in.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* context: geometry + neighbour tables                                */
/* ------------------------------------------------------------------ */

typedef struct {
  int L[4];
  long V, nEven, nOdd;
  int nlinks;           /* 4 or 8 */
  int32_t *coord;       /* [V][4] coordinates of each site index */
  int32_t *fwd;         /* [nlinks][V]: index of x + len_k * mu_k */
  int32_t *bck;         /* [nlinks][V]: index of x - len_k * mu_k */
  const double *links;  /* borrowed, [nlinks][V][18] */
  double *tmp;          /* odd temporary for stagD2ee, [V][6] */
} OCtx;

long or_index(const int L[4], const int x[4]) {
  /* qlayout.nim:108-136 with innerGeom = 1, one rank */
  long V = (long)L[0] * L[1] * L[2] * L[3];
  long lex = x[0] + (long)L[0] * (x[1] + (long)L[1] * (x[2] + (long)L[2] * x[3]));
  int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  return (lex + (p ? V : 0)) / 2;
}

void or_coords(const int L[4], int32_t *coord) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  for (long lex = 0; lex < V; lex++) {
    int x[4];
    long t = lex;
    for (int d = 0; d < 4; d++) { x[d] = (int)(t % L[d]); t /= L[d]; }
    long i = or_index(L, x);
    for (int d = 0; d < 4; d++) coord[4 * i + d] = x[d];
  }
}

static int hop_mu(int nlinks, int k) { return nlinks == 8 ? k / 2 : k; }
static int hop_len(int nlinks, int k) { return nlinks == 8 ? ((k & 1) ? 3 : 1) : 1; }

static long shifted_index(const int L[4], const int32_t *c, int mu, int len) {
  int x[4] = {c[0], c[1], c[2], c[3]};
  x[mu] = ((x[mu] + len) % L[mu] + L[mu]) % L[mu];
  return or_index(L, x);
}

/* Neighbour table of QEX's ShiftB(dir=mu, len, subset=parity): for each
   destination site i of the subset (in subset order) the index of x(i)+len*mu.
   parity: 0 even, 1 odd, 2 all sites. */
void or_shift_table(const int L[4], int mu, int len, int parity, int32_t *pidx) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  long nEven = V - V / 2;
  int32_t *coord = (int32_t *)malloc(sizeof(int32_t) * 4 * V);
  or_coords(L, coord);
  long i0 = parity == 1 ? nEven : 0;
  long i1 = parity == 0 ? nEven : V;
  for (long i = i0; i < i1; i++) pidx[i - i0] = (int32_t)shifted_index(L, coord + 4 * i, mu, len);
  free(coord);
}

void *or_ctx_create(const int L[4], int nlinks, const double *links) {
  OCtx *c = (OCtx *)calloc(1, sizeof(OCtx));
  for (int d = 0; d < 4; d++) c->L[d] = L[d];
  c->V = (long)L[0] * L[1] * L[2] * L[3];
  c->nOdd = c->V / 2;
  c->nEven = c->V - c->nOdd;
  c->nlinks = nlinks;
  c->links = links;
  c->coord = (int32_t *)malloc(sizeof(int32_t) * 4 * c->V);
  or_coords(L, c->coord);
  c->fwd = (int32_t *)malloc(sizeof(int32_t) * nlinks * c->V);
  c->bck = (int32_t *)malloc(sizeof(int32_t) * nlinks * c->V);
  for (int k = 0; k < nlinks; k++) {
    int mu = hop_mu(nlinks, k), len = hop_len(nlinks, k);
    for (long i = 0; i < c->V; i++) {
      c->fwd[k * c->V + i] = (int32_t)shifted_index(L, c->coord + 4 * i, mu, len);
      c->bck[k * c->V + i] = (int32_t)shifted_index(L, c->coord + 4 * i, mu, -len);
    }
  }
  c->tmp = (double *)calloc(6 * c->V, sizeof(double));
  return c;
}

void or_ctx_set_links(void *ctx, const double *links) { ((OCtx *)ctx)->links = links; }

void or_ctx_destroy(void *ctx) {
  OCtx *c = (OCtx *)ctx;
  if (!c) return;
  free(c->coord); free(c->fwd); free(c->bck); free(c->tmp);
  free(c);
}

/* ------------------------------------------------------------------ */
/* phases and boundary conditions                                      */
/* ------------------------------------------------------------------ */

/* Staggered phase of direction mu at coordinates x, QEX phases [8,9,11,0]
   (stagD.nim:560-571): eta_mu = (-1)^(sum_k bit_k(phases[mu]) * x_k). */
int or_stag_eta(int mu, const int x[4]) {
  static const int ph[4] = {8, 9, 11, 0};
  int s = 0;
  for (int k = 0; k < 4; k++) s += ((ph[mu] >> k) & 1) * x[k];
  return (s & 1) ? -1 : 1;
}

/* Fold phases into a link list in place.  For one-hop links this is
   setBC (negate U_3 on the last time slice, gaugeUtils.nim:133-140) followed
   by stagPhase.  For three-hop long links (k odd when nlinks==8) the sign is
   the product over the three constituent one-hop links, which is
   eta_mu(x) times -1 when the hop x -> x+3t crosses the time boundary. */
void or_apply_phases(const int L[4], int nlinks, double *links) {
  long V = (long)L[0] * L[1] * L[2] * L[3];
  int32_t *coord = (int32_t *)malloc(sizeof(int32_t) * 4 * V);
  or_coords(L, coord);
  for (int k = 0; k < nlinks; k++) {
    int mu = hop_mu(nlinks, k), len = hop_len(nlinks, k);
    for (long i = 0; i < V; i++) {
      const int32_t *xc = coord + 4 * i;
      int x[4] = {xc[0], xc[1], xc[2], xc[3]};
      int s = or_stag_eta(mu, x);
      if (mu == 3 && x[3] + len >= L[3]) s = -s;
      if (s < 0) {
        double *u = links + ((long)k * V + i) * 18;
        for (int e = 0; e < 18; e++) u[e] = -u[e];
      }
    }
  }
  free(coord);
}

/* ------------------------------------------------------------------ */
/* site algebra                                                        */
/* ------------------------------------------------------------------ */

/* r += U x */
static inline void madd_mv(double *r, const double *u, const double *x) {
  for (int i = 0; i < 3; i++) {
    double re = r[2 * i], im = r[2 * i + 1];
    for (int j = 0; j < 3; j++) {
      double ur = u[6 * i + 2 * j], ui = u[6 * i + 2 * j + 1];
      double xr = x[2 * j], xi = x[2 * j + 1];
      re += ur * xr - ui * xi;
      im += ur * xi + ui * xr;
    }
    r[2 * i] = re; r[2 * i + 1] = im;
  }
}

/* r -= U x */
static inline void msub_mv(double *r, const double *u, const double *x) {
  for (int i = 0; i < 3; i++) {
    double re = r[2 * i], im = r[2 * i + 1];
    for (int j = 0; j < 3; j++) {
      double ur = u[6 * i + 2 * j], ui = u[6 * i + 2 * j + 1];
      double xr = x[2 * j], xi = x[2 * j + 1];
      re -= ur * xr - ui * xi;
      im -= ur * xi + ui * xr;
    }
    r[2 * i] = re; r[2 * i + 1] = im;
  }
}

/* t = U^dagger x */
static inline void adj_mv(double *t, const double *u, const double *x) {
  for (int i = 0; i < 3; i++) {
    double re = 0, im = 0;
    for (int j = 0; j < 3; j++) {
      double ur = u[6 * j + 2 * i], ui = -u[6 * j + 2 * i + 1];
      double xr = x[2 * j], xi = x[2 * j + 1];
      re += ur * xr - ui * xi;
      im += ur * xi + ui * xr;
    }
    t[2 * i] = re; t[2 * i + 1] = im;
  }
}

static void subset_range(const OCtx *c, int parity, long *i0, long *i1) {
  *i0 = parity == 1 ? c->nEven : 0;
  *i1 = parity == 0 ? c->nEven : c->V;
}

/* ------------------------------------------------------------------ */
/* operators                                                           */
/* ------------------------------------------------------------------ */

/* stagD2 (stagD.nim:383-448): on the subset,
   r = a*r + b*x + sum_k [ U_k(s) x(s+d_k) - U_k(s-d_k)^dagger x(s-d_k) ]
   with, per k, the forward term added before the backward one is subtracted.
   hop_sign = -1 gives stagDM's form (stagD.nim:312-347): subtract forward,
   add backward. */
static void stagD2_core(const OCtx *c, int parity, double *r, const double *x,
                        double a, double b, int hop_sign) {
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  const long V = c->V;
  const int nl = c->nlinks;
  const double *g = c->links;
#pragma omp parallel for schedule(static)
  for (long i = i0; i < i1; i++) {
    double rir[6], t[6];
    if (a == 0 && b == 0) {
      /* stagDP's "rir := 0" (stagD.nim:502-503); also what stagD2's
         b*x gives for finite x */
      for (int e = 0; e < 6; e++) rir[e] = 0.0;
    } else if (a == 0) {
      for (int e = 0; e < 6; e++) rir[e] = b * x[6 * i + e];
    } else {
      for (int e = 0; e < 6; e++) rir[e] = a * r[6 * i + e] + b * x[6 * i + e];
    }
    for (int k = 0; k < nl; k++) {
      long jf = c->fwd[k * V + i];
      long jb = c->bck[k * V + i];
      const double *uf = g + ((long)k * V + i) * 18;
      const double *ub = g + ((long)k * V + jb) * 18;
      adj_mv(t, ub, x + 6 * jb);
      if (hop_sign > 0) {
        madd_mv(rir, uf, x + 6 * jf);
        for (int e = 0; e < 6; e++) rir[e] -= t[e];
      } else {
        msub_mv(rir, uf, x + 6 * jf);
        for (int e = 0; e < 6; e++) rir[e] += t[e];
      }
    }
    for (int e = 0; e < 6; e++) r[6 * i + e] = rir[e];
  }
}

void or_stagD2(void *ctx, int parity, double *r, const double *x, double a, double b) {
  stagD2_core((const OCtx *)ctx, parity, r, x, a, b, 1);
}

/* stagD (stagD.nim:459-462): r = a*r + m*x + (sc/2)(2D)x on the subset,
   computed as stagD2 with a/(sc/2), m/(sc/2) then a final scale by sc/2. */
void or_stagD(void *ctx, int parity, double *r, const double *x, double m, double sc, double a) {
  const OCtx *c = (const OCtx *)ctx;
  double h = 0.5 * sc;
  stagD2_core(c, parity, r, x, a / h, m / h, 1);
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
#pragma omp parallel for schedule(static)
  for (long i = 6 * i0; i < 6 * i1; i++) r[i] *= h;
}

/* D and Ddag (stagD.nim:617-622): even then odd subsets. */
void or_D(void *ctx, double *r, const double *x, double m) {
  or_stagD(ctx, 0, r, x, m, 1.0, 0.0);
  or_stagD(ctx, 1, r, x, m, 1.0, 0.0);
}
void or_Ddag(void *ctx, double *r, const double *x, double m) {
  or_stagD(ctx, 0, r, x, m, -1.0, 0.0);
  or_stagD(ctx, 1, r, x, m, -1.0, 0.0);
}

/* stagDM (stagD.nim:312-347) with the init expression of stagD2xx
   (rir := 4 m2 x, stagD.nim:508-509): the init reads x while the hopping
   input is the temporary t, so r = 4 m2 x - (2D) t, per k the forward term
   subtracted then the backward term added. */
static void stagDM_init(const OCtx *c, int parity, double *r, const double *t,
                        const double *x, double init) {
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  const long V = c->V;
  const int nl = c->nlinks;
  const double *g = c->links;
#pragma omp parallel for schedule(static)
  for (long i = i0; i < i1; i++) {
    double rir[6], w[6];
    for (int e = 0; e < 6; e++) rir[e] = init * x[6 * i + e];
    for (int k = 0; k < nl; k++) {
      long jf = c->fwd[k * V + i];
      long jb = c->bck[k * V + i];
      const double *uf = g + ((long)k * V + i) * 18;
      const double *ub = g + ((long)k * V + jb) * 18;
      msub_mv(rir, uf, t + 6 * jf);
      adj_mv(w, ub, t + 6 * jb);
      for (int e = 0; e < 6; e++) rir[e] += w[e];
    }
    for (int e = 0; e < 6; e++) r[6 * i + e] = rir[e];
  }
}

/* stagD2xx (stagD.nim:485-512): t_y = (2D)_yx x_x (stagDP with rir := 0),
   then r_x = 4 m2 x_x - (2D)_xy t_y.  parity selects x (0 even = stagD2ee). */
void or_stagD2ee_par(void *ctx, int parity, double *r, const double *x, double m2) {
  OCtx *c = (OCtx *)ctx;
  stagD2_core(c, 1 - parity, c->tmp, x, 0.0, 0.0, 1);
  stagDM_init(c, parity, r, c->tmp, x, 4.0 * m2);
}
void or_stagD2ee(void *ctx, double *r, const double *x, double m2) { or_stagD2ee_par(ctx, 0, r, x, m2); }
void or_stagD2oo(void *ctx, double *r, const double *x, double m2) { or_stagD2ee_par(ctx, 1, r, x, m2); }

/* ------------------------------------------------------------------ */
/* field reductions on a subset (fieldET.nim:648-780)                  */
/* ------------------------------------------------------------------ */

static double norm2_sub(const OCtx *c, int parity, const double *x) {
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 6 * i0; i < 6 * i1; i++) s += x[i] * x[i];
  return s;
}
static double redot_sub(const OCtx *c, int parity, const double *x, const double *y) {
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 6 * i0; i < 6 * i1; i++) s += x[i] * y[i];
  return s;
}
double or_norm2(void *ctx, int parity, const double *x) { return norm2_sub((OCtx *)ctx, parity, x); }
double or_redot(void *ctx, int parity, const double *x, const double *y) {
  return redot_sub((OCtx *)ctx, parity, x, y);
}

/* ------------------------------------------------------------------ */
/* CG (cg.nim:55-272, precon cpNone) on one parity for                  */
/*   A y = b, A = stagD2xx(m2); x enters as the initial guess.          */
/* ------------------------------------------------------------------ */

/* The solve is split into begin / run / end so that a caller can run it in
   bounded pieces (the CPU baseline times one whole solve as a sequence of
   steps); or_cg_xx is begin, one run to maxits, end. */
typedef struct {
  OCtx *c;
  int parity;
  long i0, i1;
  double *x, *r, *p, *Ap;
  double m2, b2, r2, rzo, r2stop;
  int itn;
} OrCg;

void *or_cg_begin(void *ctx, int parity, double *x, const double *b, double m2, double r2req) {
  OCtx *c = (OCtx *)ctx;
  OrCg *s = (OrCg *)calloc(1, sizeof(OrCg));
  long n = 6 * c->V;
  s->c = c;
  s->parity = parity;
  subset_range(c, parity, &s->i0, &s->i1);
  s->x = x;
  s->m2 = m2;
  s->r = (double *)calloc(n, sizeof(double));
  s->p = (double *)calloc(n, sizeof(double));
  s->Ap = (double *)calloc(n, sizeof(double));
  s->b2 = norm2_sub(c, parity, b);
  s->r2 = 0;
  s->rzo = 1.0;
  s->itn = 0;
  if (s->b2 == 0.0) {
    for (long i = 6 * s->i0; i < 6 * s->i1; i++) x[i] = 0;
  } else {
    or_stagD2ee_par(c, parity, s->Ap, x, m2);
    for (long i = 6 * s->i0; i < 6 * s->i1; i++) { s->r[i] = b[i] - s->Ap[i]; s->p[i] = 0; }
    s->r2 = norm2_sub(c, parity, s->r);
  }
  s->r2stop = r2req * s->b2;
  return s;
}

/* Runs iterations until itn reaches maxits (a total, not a count for this
   call) or the residual meets the target; returns itn. */
int or_cg_run(void *state, int maxits) {
  OrCg *s = (OrCg *)state;
  OCtx *c = s->c;
  const long i0 = s->i0, i1 = s->i1;
  double *x = s->x, *r = s->r, *p = s->p, *Ap = s->Ap;
  while (s->itn < maxits && s->r2 > s->r2stop) {
    double rz = s->r2;
    double beta = rz / s->rzo;
    s->rzo = rz;
    if (s->itn == 0) {
      for (long i = 6 * i0; i < 6 * i1; i++) p[i] = r[i];
    } else {
      for (long i = 6 * i0; i < 6 * i1; i++) p[i] = r[i] + beta * p[i];
    }
    s->itn++;
    or_stagD2ee_par(c, s->parity, Ap, p, s->m2);
    double pAp = redot_sub(c, s->parity, p, Ap);
    double alpha = rz / pAp;
#pragma omp parallel for schedule(static)
    for (long i = 6 * i0; i < 6 * i1; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    s->r2 = norm2_sub(c, s->parity, r);
  }
  return s->itn;
}

/* 1 once the iterated residual meets the target. */
int or_cg_converged(void *state) {
  OrCg *s = (OrCg *)state;
  return !(s->r2 > s->r2stop);
}

/* Frees the state; returns the iterations and *r2_out = |r|^2/|b|^2. */
int or_cg_end(void *state, double *r2_out) {
  OrCg *s = (OrCg *)state;
  int itn = s->itn;
  if (r2_out) *r2_out = (s->b2 > 0) ? s->r2 / s->b2 : 0.0;
  free(s->r); free(s->p); free(s->Ap);
  free(s);
  return itn;
}

int or_cg_xx(void *ctx, int parity, double *x, const double *b, double m2,
             double r2req, int maxits, double *r2_out) {
  void *s = or_cg_begin(ctx, parity, x, b, m2, r2req);
  or_cg_run(s, maxits);
  return or_cg_end(s, r2_out);
}

/* solveXXInternal for the FP64 QEX backend (stagSolve.nim:90-161 and
   60-88): the solution is zeroed, then CG runs from zero. */
static int solveXXInternal(OCtx *c, int parity, double *y, const double *b, double m,
                           double r2req, int maxits) {
  long n = 6 * c->V;
  memset(y, 0, sizeof(double) * n);
  return or_cg_xx(c, parity, y, b, m * m, r2req, maxits, NULL);
}

/* solveXX (stagSolve.nim:330-421): defect correction around the inner
   solve.  Solves stagD2xx(m^2) r = x on the parity; r is zeroed first.
   Returns total iterations; *r2_out = final true |rho|^2/|b|^2. */
int or_solveXX(void *ctx, int parity, double *r, const double *x, double m,
               double r2req, int maxits, double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  long n = 6 * c->V;
  double *rho = (double *)calloc(n, sizeof(double));
  double *y = (double *)calloc(n, sizeof(double));
  memset(r, 0, sizeof(double) * n);
  for (long i = 6 * i0; i < 6 * i1; i++) rho[i] = x[i];
  double b2 = norm2_sub(c, parity, rho);
  double r2 = b2, r2Stop = r2req * b2, r2Prev = INFINITY;
  int its = 0;
  while (r2 > r2Stop && r2 < r2Prev) {
    r2Prev = r2;
    int mx = maxits - its;
    if (mx <= 0) break;
    its += solveXXInternal(c, parity, y, rho, m, r2Stop / r2, mx);
    for (long i = 6 * i0; i < 6 * i1; i++) r[i] += y[i];
    or_stagD2ee_par(c, parity, rho, r, m * m);
    for (long i = 6 * i0; i < 6 * i1; i++) rho[i] = x[i] - rho[i];
    r2 = norm2_sub(c, parity, rho);
  }
  if (r2_out) *r2_out = b2 > 0 ? r2 / b2 : 0.0;
  free(rho); free(y);
  return its;
}

/* eoReconstruct (stagD.nim:633-637): r_o = (b_o - D_oe r_e)/m. */
void or_eoReconstruct(void *ctx, double *r, const double *b, double m) {
  OCtx *c = (OCtx *)ctx;
  or_stagD(c, 1, r, r, 0.0, -1.0 / m, 0.0);
#pragma omp parallel for schedule(static)
  for (long i = 6 * c->nEven; i < 6 * c->V; i++) r[i] += b[i] / m;
}

/* solveReconR / solveReconL / solveInner (stagSolve.nim:238-326). */
static int solveReconR(OCtx *c, double *x, const double *b, double m, double r2req,
                       int maxits, double b2e, double b2o) {
  long n = 6 * c->V;
  double b2 = b2e + b2o;
  double r2stop = r2req * b2, r2stop2 = 0.5 * r2stop;
  double r2stope = (b2o <= r2stop2) ? r2stop - b2o : r2stop2;
  double *y = (double *)calloc(n, sizeof(double));
  int its = 0;
  if (b2e > r2stope) {
    its = solveXXInternal(c, 0, y, b, m, r2stope / b2e, maxits);
    for (long i = 0; i < 6 * c->nEven; i++) y[i] *= 4;
    or_Ddag(c, x, y, m);
    free(y);
    return its;
  }
  double r2stopo = (b2e <= r2stop2) ? r2stop - b2e : r2stop2;
  if (b2o > r2stopo) {
    its = solveXXInternal(c, 1, y, b, m, r2stopo / b2o, maxits);
    for (long i = 6 * c->nEven; i < n; i++) y[i] *= 4;
    or_Ddag(c, x, y, m);
  }
  free(y);
  return its;
}

static int solveReconL(OCtx *c, double *x, const double *b, double m, double r2req,
                       int maxits, double b2e, double b2o) {
  long n = 6 * c->V;
  double *d = (double *)calloc(n, sizeof(double));
  or_Ddag(c, d, b, m);
  memset(x, 0, sizeof(double) * n);
  double d2e = norm2_sub(c, 0, d);
  double req = 0.99 * r2req * (b2e + b2o) * m * m / d2e;
  int its = solveXXInternal(c, 0, x, d, m, req, maxits);
  for (long i = 0; i < 6 * c->nEven; i++) x[i] *= 4;
  or_eoReconstruct(c, x, b, m);
  free(d);
  return its;
}

static int solveInner(OCtx *c, double *x, const double *b, double m, double r2req,
                      int maxits, double b2e, double b2o) {
  double b2 = b2e + b2o;
  double r2stop = r2req * b2, r2stop2 = 0.5 * r2stop;
  double r2stope = (b2o <= r2stop2) ? r2stop - b2o : r2stop2;
  double r2stopo = (b2e <= r2stop2) ? r2stop - b2e : r2stop2;
  if (b2e <= r2stope || b2o <= r2stopo || m == 0.0)
    return solveReconR(c, x, b, m, r2req, maxits, b2e, b2o);
  return solveReconL(c, x, b, m, r2req, maxits, b2e, b2o);
}

/* solve (stagSolve.nim:469-557): D(m) x = b on the full lattice, x zeroed
   (usePrevSoln false).  Returns iterations; *r2_out = |b - D x|^2/|b|^2. */
int or_solve(void *ctx, double *x, const double *b, double m, double r2req, int maxits,
             double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  long n = 6 * c->V;
  double b2 = norm2_sub(c, 2, b);
  double r2stop = r2req * b2;
  double *r = (double *)malloc(sizeof(double) * n);
  double *y = (double *)calloc(n, sizeof(double));
  memset(x, 0, sizeof(double) * n);
  memcpy(r, b, sizeof(double) * n);
  double r2e = norm2_sub(c, 0, r), r2o = norm2_sub(c, 1, r);
  double r2 = r2e + r2o;
  int its = 0;
  while (r2 > r2stop) {
    int mx = maxits - its;
    if (mx <= 0) break;
    double req = r2stop / r2;
    memset(y, 0, sizeof(double) * n);
    its += solveInner(c, y, r, m, req, mx, r2e, r2o);
    for (long i = 0; i < n; i++) x[i] += y[i];
    or_D(c, r, x, m);
    for (long i = 0; i < n; i++) r[i] = b[i] - r[i];
    r2e = norm2_sub(c, 0, r);
    r2o = norm2_sub(c, 1, r);
    r2 = r2e + r2o;
  }
  if (r2_out) *r2_out = b2 > 0 ? r2 / b2 : 0.0;
  free(r); free(y);
  return its;
}

/* ------------------------------------------------------------------ */
/* multi-shift CG (cgm.nim:68-246) on one parity:                       */
/*   (A + sg[k]) xs[k] = b, A = stagD2xx(m2), sg[0] must be 0.          */
/* xs: nshift pointers to full fields; zeroed here (fresh solve).       */
/* ------------------------------------------------------------------ */

int or_cgm_xx(void *ctx, int parity, int nshift, double **xs, const double *sg_in,
              const double *b, double m2, double r2req, int maxits, double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  long i0, i1;
  subset_range(c, parity, &i0, &i1);
  long n = 6 * c->V;
  double *r = (double *)calloc(n, sizeof(double));
  double *Ap = (double *)calloc(n, sizeof(double));
  double **ps = (double **)malloc(sizeof(double *) * nshift);
  double *sg = (double *)malloc(sizeof(double) * nshift);
  double *zi = (double *)malloc(sizeof(double) * nshift);
  double *zim1 = (double *)malloc(sizeof(double) * nshift);
  for (int k = 0; k < nshift; k++) {
    ps[k] = (double *)calloc(n, sizeof(double));
    sg[k] = (k == 0) ? 0.0 : sg_in[k];
  }
  for (long i = 6 * i0; i < 6 * i1; i++) r[i] = b[i];
  for (int k = 0; k < nshift; k++)
    for (long i = 6 * i0; i < 6 * i1; i++) xs[k][i] = 0;
  double b2 = norm2_sub(c, parity, b);
  double r2 = b2;
  double r2stop = r2req * b2;
  int itn = 0;
  if (r2 > r2stop) {
    double r2i = r2, r2ip1 = 0, r2r = 0, pAp, alpha = 0, beta = 0;
    double alphaim1 = -1.0, betaim1 = 0.0;
    int continuing = 1;
    for (int k = 0; k < nshift; k++) {
      zim1[k] = 1.0; zi[k] = 1.0;
      for (long i = 6 * i0; i < 6 * i1; i++) ps[k][i] = r[i];
    }
    while (continuing) {
      for (int k = 0; k < nshift; k++) {
        if (k == 0) {
          or_stagD2ee_par(c, parity, Ap, ps[0], m2);
          itn++;
          pAp = redot_sub(c, parity, ps[0], Ap);
          alpha = (pAp != 0.0) ? r2i / pAp : 0.0;
#pragma omp parallel for schedule(static)
          for (long i = 6 * i0; i < 6 * i1; i++) {
            r[i] -= alpha * Ap[i];
            xs[0][i] += alpha * ps[0][i];
          }
          r2ip1 = norm2_sub(c, parity, r);
          r2r = r2ip1;
          beta = (r2i != 0.0) ? r2ip1 / r2i : 0.0;
          continuing = (itn < maxits) && (r2r > r2stop);
          if (continuing)
            for (long i = 6 * i0; i < 6 * i1; i++) ps[0][i] = r[i] + beta * ps[0][i];
        } else {
          double zip1d = alpha * betaim1 * (zim1[k] - zi[k]);
          zip1d += zim1[k] * alphaim1 * (1.0 + sg[k] * alpha);
          double zip1 = (zip1d != 0.0) ? zi[k] * zim1[k] * alphaim1 / zip1d : 0.0;
          double zr = (zi[k] != 0.0) ? zip1 / zi[k] : 0.0;
          double az = alpha * zr;
          for (long i = 6 * i0; i < 6 * i1; i++) xs[k][i] += az * ps[k][i];
          if (continuing) {
            double bz = beta * zr * zr;
            for (long i = 6 * i0; i < 6 * i1; i++) ps[k][i] = zip1 * r[i] + bz * ps[k][i];
            zim1[k] = zi[k];
            zi[k] = zip1;
          }
        }
      }
      alphaim1 = alpha;
      betaim1 = beta;
      r2i = r2ip1;
      r2 = r2r;
    }
  }
  if (r2_out) *r2_out = b2 > 0 ? r2 / b2 : 0.0;
  for (int k = 0; k < nshift; k++) free(ps[k]);
  free(ps); free(sg); free(zi); free(zim1); free(r); free(Ap);
  return itn;
}

/* multi-mass solve (stagSolve.nim:560-668): D(ms[k]) xs[k] = b for all k
   from one multi-shift CG per outer pass on the parity whose residual is
   large, shifts 4(ms[k]^2 - ms[0]^2), then xs[k] = Ddag(ms[k]) (4 y_k).
   Returns iterations; *r2_out = final |b - D(ms[0]) Ddag(ms[0]) 4y_0|^2/|b|^2. */
int or_solve_multishift(void *ctx, int nmass, double **xs, const double *b, const double *ms,
                        double r2req, int maxits, double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  long n = 6 * c->V;
  double mass = ms[0];
  double b2e = norm2_sub(c, 0, b), b2o = norm2_sub(c, 1, b);
  double b2 = b2e + b2o;
  double r2 = b2e + b2o;
  double r2stop = r2req * b2;
  double *r = (double *)malloc(sizeof(double) * n);
  double *xt = (double *)calloc(n, sizeof(double));
  double *shifts = (double *)malloc(sizeof(double) * nmass);
  double **ys = (double **)malloc(sizeof(double *) * nmass);
  memcpy(r, b, sizeof(double) * n);
  for (int k = 0; k < nmass; k++) {
    shifts[k] = (k == 0) ? ms[0] : 4.0 * (ms[k] * ms[k] - mass * mass);
    ys[k] = (double *)calloc(n, sizeof(double));
    memset(xs[k], 0, sizeof(double) * n);
  }
  int its = 0;
  while (r2 > r2stop) {
    int mx = maxits - its;
    if (mx <= 0) break;
    double req = r2stop;
    double r2stop2 = 0.5 * req;
    double r2stope = (b2o <= r2stop2) ? req - b2o : r2stop2;
    double r2stopo = (b2e <= r2stop2) ? req - b2e : r2stop2;
    int par;
    if (b2e > r2stope) { req = r2stope / b2e; par = 0; }
    else if (b2o > r2stopo) { req = r2stopo / b2o; par = 1; }
    else break;
    its += or_cgm_xx(c, par, nmass, ys, shifts, r, mass * mass, req, mx, NULL);
    long i0 = par ? 6 * c->nEven : 0, i1 = par ? n : 6 * c->nEven;
    for (int k = 0; k < nmass; k++)
      for (long i = i0; i < i1; i++) xs[k][i] += 4.0 * ys[k][i];
    or_Ddag(c, xt, xs[0], mass);
    or_D(c, r, xt, mass);
    for (long i = 0; i < n; i++) r[i] = b[i] - r[i];
    b2e = norm2_sub(c, 0, r);
    b2o = norm2_sub(c, 1, r);
    r2 = b2e + b2o;
  }
  double *t2 = (double *)malloc(sizeof(double) * n);
  for (int k = 0; k < nmass; k++) {
    if (k != 0) or_Ddag(c, xt, xs[k], ms[k]);
    memcpy(t2, xt, sizeof(double) * n);
    memcpy(xs[k], t2, sizeof(double) * n);
  }
  if (r2_out) *r2_out = b2 > 0 ? r2 / b2 : 0.0;
  for (int k = 0; k < nmass; k++) free(ys[k]);
  free(ys); free(shifts); free(r); free(xt); free(t2);
  return its;
}

/* ------------------------------------------------------------------ */
/* fermion force (hmcAction.nim:669-790, no smearing)                   */
/* ------------------------------------------------------------------ */

/* projectTAH (matrixFunctions.nim:414-419): traceless anti-Hermitian part,
   r = (m - m^dagger)/2 - Tr((m - m^dagger)/2)/3. */
void or_project_tah(double *r, const double *m) {
  double t[18];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      t[6 * i + 2 * j] = 0.5 * (m[6 * i + 2 * j] - m[6 * j + 2 * i]);
      t[6 * i + 2 * j + 1] = 0.5 * (m[6 * i + 2 * j + 1] + m[6 * j + 2 * i + 1]);
    }
  double tri = (t[1] + t[9] + t[17]) / 3.0;
  t[1] -= tri; t[9] -= tri; t[17] -= tri;
  memcpy(r, t, sizeof(t));
}

/* stagForceSolve (hmcAction.nim:669-721): solveEE(varphi, phi, mass),
   varphi_e *= 4, psi_o = (2D)_oe varphi_e (stagD2 with a = b = 0),
   psi_e = varphi_e.  Returns iterations. */
int or_force_solve(void *ctx, double *psi, const double *phi, double m, double r2req,
                   int maxits, double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  long n = 6 * c->V;
  double *varphi = (double *)calloc(n, sizeof(double));
  memset(psi, 0, sizeof(double) * n);
  int its = or_solveXX(c, 0, varphi, phi, m, r2req, maxits, r2_out);
  for (long i = 0; i < 6 * c->nEven; i++) varphi[i] *= 4.0;
  stagD2_core(c, 1, psi, varphi, 0.0, 0.0, 1);
  for (long i = 0; i < 6 * c->nEven; i++) psi[i] = varphi[i];
  free(varphi);
  return its;
}

/* fermForce (hmcAction.nim:723-790) without smearing, generalised to the
   link list: for link k with hop len along mu,
     f1_k(x)[a,b] = psi_a(x) conj(psi_b(x + len mu)), negated on odd x,
     f_k(x) = projectTAH(f1_k(x) U_k(x)^dagger).
   f: [nlinks][V][18]. */
void or_ferm_force(void *ctx, double *f, const double *psi) {
  OCtx *c = (OCtx *)ctx;
  const long V = c->V;
  const int nl = c->nlinks;
  for (int k = 0; k < nl; k++) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < V; i++) {
      const double *a = psi + 6 * i;
      const double *bb = psi + 6 * (long)c->fwd[k * V + i];
      double f1[18], m[18];
      double s = (i >= c->nEven) ? -1.0 : 1.0;
      for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
          double ar = a[2 * p], ai = a[2 * p + 1], br = bb[2 * q], bi = -bb[2 * q + 1];
          f1[6 * p + 2 * q] = s * (ar * br - ai * bi);
          f1[6 * p + 2 * q + 1] = s * (ar * bi + ai * br);
        }
      const double *u = c->links + ((long)k * V + i) * 18;
      /* m = f1 * u^dagger */
      for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
          double re = 0, im = 0;
          for (int j = 0; j < 3; j++) {
            double xr = f1[6 * p + 2 * j], xi = f1[6 * p + 2 * j + 1];
            double yr = u[6 * q + 2 * j], yi = -u[6 * q + 2 * j + 1];
            re += xr * yr - xi * yi;
            im += xr * yi + xi * yr;
          }
          m[6 * p + 2 * q] = re;
          m[6 * p + 2 * q + 1] = im;
        }
      or_project_tah(f + ((long)k * V + i) * 18, m);
    }
  }
}

/* fermForce's outer products alone (hmcAction.nim:744-771): for link k,
   f_k(x)[a,b] = s(x) psi_a(x) conj(psi_b(x + len mu)), s = -1 on odd x. */
void or_ferm_outer(void *ctx, double *f, const double *psi) {
  OCtx *c = (OCtx *)ctx;
  const long V = c->V;
  for (int k = 0; k < c->nlinks; k++) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < V; i++) {
      const double *a = psi + 6 * i;
      const double *bb = psi + 6 * (long)c->fwd[k * V + i];
      double s = (i >= c->nEven) ? -1.0 : 1.0;
      double *o = f + ((long)k * V + i) * 18;
      for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
          double ar = a[2 * p], ai = a[2 * p + 1], br = bb[2 * q], bi = -bb[2 * q + 1];
          o[6 * p + 2 * q] = s * (ar * br - ai * bi);
          o[6 * p + 2 * q + 1] = s * (ar * bi + ai * br);
        }
    }
  }
}

/* stagForceSolve followed by fermForce: the force QEX's
   StaggeredFermionAction.force hands to addForce (before its 0.25*dtau). */
int or_force(void *ctx, double *f, const double *phi, double m, double r2req, int maxits,
             double *r2_out) {
  OCtx *c = (OCtx *)ctx;
  double *psi = (double *)calloc(6 * c->V, sizeof(double));
  int its = or_force_solve(c, psi, phi, m, r2req, maxits, r2_out);
  or_ferm_force(c, f, psi);
  free(psi);
  return its;
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
