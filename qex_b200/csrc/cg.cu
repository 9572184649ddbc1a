// cg.cu -- FP64 conjugate gradient (src/solvers/cg.nim:55-272, precon
// cpNone) on one parity of the Schur operator, with every scalar kept on the
// device: the host only enqueues iterations and reads the CgState every few
// iterations to see whether the solve is done.  Kernels launched after
// convergence return at once (CgState.done), so the iteration count and the
// solution are those of QEX's loop
//   while itn < maxits and r2 > r2stop:
//     beta = rz/rzo; p = (itn == 0) ? r : r + beta p; itn++
//     Ap = A p; alpha = rz/<p,Ap>; x += alpha p; r -= alpha Ap; r2 = |r|^2
// Also the solve drivers solveXX (stagSolve.nim:330-421) and solve
// (stagSolve.nim:469-557, with solveInner/solveReconL/solveReconR).
#include <chrono>
#include <cmath>
#include <cstring>

#include "lib.cuh"

namespace qs {

int cg_mixed(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits,
             int sloppy, double delta, CgOut *out, int *reliable);

__global__ void __launch_bounds__(kBlock)
    cg_init_kernel(const double2 *__restrict__ b, int bs, double2 *__restrict__ r, int rs,
                   double2 *__restrict__ x, int xs, int n, CgState *st, double *partials,
                   unsigned *ticket) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 v = b[(size_t)c * bs + i];
      r[(size_t)c * rs + i] = v;
      x[(size_t)c * xs + i] = make_double2(0.0, 0.0);
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) {
    double b2 = o[0];
    st->b2 = b2;
    st->r2 = b2;
    st->rz = b2;
    st->r2stop = st->r2req * b2;
    st->itn = 0;
    st->beta = 0.0;
    st->nan = isnan(b2) ? 1 : 0;
    st->done = (!(b2 > st->r2stop) || st->maxits <= 0 || st->nan) ? 1 : 0;
  }
}

__global__ void cg_p_kernel(const double2 *__restrict__ r, int rs, double2 *__restrict__ p, int ps,
                            int n, const CgState *st) {
  pdl_wait();
  if (st->done) return;
  const bool first = (st->itn == 0);
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 rv = r[(size_t)c * rs + i];
      double2 o;
      if (first) {
        o = rv;
      } else {
        double2 pv = p[(size_t)c * ps + i];
        o = make_double2(fma(beta, pv.x, rv.x), fma(beta, pv.y, rv.y));
      }
      p[(size_t)c * ps + i] = o;
    }
  }
}

__global__ void __launch_bounds__(kBlock)
    cg_xr_kernel(double2 *__restrict__ x, int xs, double2 *__restrict__ r, int rs,
                 const double2 *__restrict__ p, int ps, const double2 *__restrict__ ap, int aps,
                 int n, CgState *st, double *partials, unsigned *ticket) {
  pdl_wait();
  if (st->done) return;
  const double alpha = st->alpha;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 pv = p[(size_t)c * ps + i], av = ap[(size_t)c * aps + i];
      double2 xv = x[(size_t)c * xs + i], rv = r[(size_t)c * rs + i];
      xv.x = fma(alpha, pv.x, xv.x);
      xv.y = fma(alpha, pv.y, xv.y);
      rv.x = fma(-alpha, av.x, rv.x);
      rv.y = fma(-alpha, av.y, rv.y);
      x[(size_t)c * xs + i] = xv;
      r[(size_t)c * rs + i] = rv;
      s = fma(rv.x, rv.x, s);
      s = fma(rv.y, rv.y, s);
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) {
    double r2 = o[0];
    st->r2 = r2;
    st->beta = r2 / st->rz;
    st->rz = r2;
    if (isnan(r2)) st->nan = 1;
    st->done = (!(st->itn < st->maxits && r2 > st->r2stop) || st->nan) ? 1 : 0;
  }
}

static_assert(sizeof(CgState) <= sizeof(double) * kNumResults, "state too large for the staging buffer");

int write_state(CgState *dst, const CgState &host) {
  double *h = host_results();
  std::memcpy(h, &host, sizeof(CgState));
  QS_CUDA(cudaMemcpyAsync(dst, h, sizeof(CgState), cudaMemcpyHostToDevice, stream()));
  return QEXSTAG_OK;
}

StateSnapshot::~StateSnapshot() {
  if (ev) cudaEventDestroy(ev);
}
int StateSnapshot::start(const void *dev, size_t bytes) {
  if (bytes > sizeof(double) * kNumResults) return fail(QEXSTAG_ERR_ARG, "state snapshot too large");
  if (!ev) QS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  QS_CUDA(cudaMemcpyAsync(host_results(), dev, bytes, cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaEventRecord(ev, stream()));
  return QEXSTAG_OK;
}
int StateSnapshot::wait(void *host, size_t bytes) {
  QS_CUDA(cudaEventSynchronize(ev));
  std::memcpy(host, host_results(), bytes);
  return QEXSTAG_OK;
}

// iterations enqueued between host checks: small lattices run many
// iterations per check (launch-bound), large ones few (each is long)
int check_interval(int nh) {
  if (nh <= 1 << 14) return 64;
  if (nh <= 1 << 17) return 16;
  return 8;  // 16 or 32 change a 32^4 16-bit solve by <= 1 %
}

int cg64(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits,
         CgOut *out) {
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  Workspace &ws = g->ws;
  void *pr, *pp, *pap, *pt, *pst;
  const size_t vb = sizeof(double2) * 3 * (size_t)nh;
  int rc;
  if ((rc = ws.get(kSlotCgR, vb, &pr)) || (rc = ws.get(kSlotCgP, vb, &pp)) ||
      (rc = ws.get(kSlotCgAp, vb, &pap)) || (rc = ws.get(kSlotCgT, vb, &pt)) ||
      (rc = ws.get(kSlotCgState, sizeof(CgState), &pst)))
    return rc;
  VecD r{(double2 *)pr, nh}, p{(double2 *)pp, nh}, ap{(double2 *)pap, nh}, t{(double2 *)pt, nh};
  CgState *st = (CgState *)pst;
  CgState hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.r2req = r2req;
  hs.maxits = maxits;
  if ((rc = write_state(st, hs))) return rc;
  const int grid = grid_for(nh, kBlock, 4);
  cg_init_kernel<<<grid, kBlock, 0, stream()>>>(b.p, b.stride, r.p, r.stride, x.p, x.stride, nh,
                                                st, red_partials(), red_tickets());
  note_launch();
  QS_LAUNCH_CHECK();
  const int every = check_interval(nh);
  const int pgrid = grid_for(nh, kBlock, 8);
  auto batch = [&]() -> int {
    for (int i = 0; i < every; i++) {
      launch_pdl(cg_p_kernel, pgrid, kBlock, (const double2 *)r.p, r.stride, p.p, p.stride, nh,
                 (const CgState *)st);
      note_launch();
      int rc2 = schur64(g, par, ap, cv(p), t, m2, kRedCgPAp, st, &st->done);
      if (rc2) return rc2;
      launch_pdl(cg_xr_kernel, grid, kBlock, x.p, x.stride, r.p, r.stride, (const double2 *)p.p, p.stride,
                 (const double2 *)ap.p, ap.stride, nh, st, red_partials(), red_tickets());
      note_launch();
    }
    QS_LAUNCH_CHECK();
    return QEXSTAG_OK;
  };
  // The state is read one batch behind: the next batch is queued before
  // the host waits for the snapshot, so the GPU does not idle during the
  // check; once the solve is done that batch's kernels return at once.
  StateSnapshot snap;
  if ((rc = batch())) return rc;
  for (;;) {
    if ((rc = snap.start(st, sizeof(CgState))) || (rc = batch()) || (rc = snap.wait(&hs, sizeof(CgState))))
      return rc;
    if (hs.done) break;
  }
  out->iterations = hs.itn;
  out->r2 = hs.b2 > 0 ? hs.r2 / hs.b2 : 0.0;
  out->nan = hs.nan;
  if (hs.nan) return fail(QEXSTAG_ERR_NAN, "cg: NaN in residual");
  return QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// solveXX: defect correction (stagSolve.nim:330-421)
// ---------------------------------------------------------------------------

static int inner_solve(qexstag_links_s *g, int par, double m, CVecD rho, VecD y, double r2req,
                       int maxits, const qexstag_solver_params *p, qexstag_solver_stats *st) {
  CgOut o{};
  int rc;
  if (p->sloppy == QEXSTAG_SLOPPY_NONE) {
    rc = cg64(g, par, m * m, rho, y, r2req, maxits, &o);
  } else {
    int rel = 0;
    // reliable-update threshold: with 16-bit links a residual drop of 0.3
    // between updates minimises the time (32^4, m = 0.01: 2754 iterations and
    // 0.413 s at 0.3, 3082 and 0.455 s at 0.1, 6439 at 0.02); FP32 is
    // insensitive to it and keeps 0.1
    double delta = p->delta > 0 ? p->delta : (p->sloppy == QEXSTAG_SLOPPY_HALF ? 0.3 : 0.1);
    rc = cg_mixed(g, par, m * m, rho, y, r2req, maxits, p->sloppy, delta, &o, &rel);
    st->reliable_updates += rel;
  }
  st->iterations += o.iterations;
  return rc;
}

int solve_xx(qexstag_links_s *g, int par, double2 *r, const double2 *x, double m,
             const qexstag_solver_params *p, qexstag_solver_stats *st) {
  const Geom &geo = g->l->g;
  const int nh = geo.nh;
  Workspace &ws = g->ws;
  void *prho, *py, *pt;
  const size_t vb = sizeof(double2) * 3 * (size_t)nh;
  int rc;
  if ((rc = ws.get(kSlotDcRho, vb, &prho)) || (rc = ws.get(kSlotDcY, vb, &py)) ||
      (rc = ws.get(kSlotTmpOdd, vb, &pt)))
    return rc;
  VecD rho{(double2 *)prho, nh}, y{(double2 *)py, nh}, t{(double2 *)pt, nh};
  VecD rpar = block(r, geo, par);
  CVecD xpar = block(x, geo, par);
  // r := 0 on all sites, rho[par] := x
  if ((rc = vzero(VecD{r, geo.V}, geo.V))) return rc;
  if ((rc = vcopy(rho, xpar, nh))) return rc;
  double b2 = 0;
  if ((rc = vnorm2(cv(rho), nh, &b2))) return rc;
  if (!std::isfinite(b2)) return fail(QEXSTAG_ERR_NAN, "solveXX: source is not finite");
  double r2 = b2, r2stop = p->r2req * b2, r2prev = INFINITY;
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  while (r2 > r2stop && r2 < r2prev) {
    r2prev = r2;
    int mx = maxits - st->iterations;
    if (mx <= 0) break;
    if ((rc = inner_solve(g, par, m, cv(rho), y, r2stop / r2, mx, p, st))) return rc;
    st->outer_iterations += 1;
    if ((rc = vaxpy(rpar, 1.0, cv(y), nh))) return rc;
    if ((rc = schur64(g, par, rho, cv(rpar), t, m * m))) return rc;
    if ((rc = vsub(rho, xpar, cv(rho), nh))) return rc;
    if ((rc = vnorm2(cv(rho), nh, &r2))) return rc;
    if (std::isnan(r2)) return fail(QEXSTAG_ERR_NAN, "solveXX: NaN residual");
  }
  st->r2 = b2 > 0 ? r2 / b2 : 0.0;
  return (r2 > r2stop) ? QEXSTAG_NOT_CONVERGED : QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// solve: full-lattice D(m) x = b (stagSolve.nim:469-557)
// ---------------------------------------------------------------------------

// stagD on one parity: r = a r + m x + (sc/2)(2D)x (stagD.nim:459-462)
int stagD_par(qexstag_links_s *g, int par, double2 *r, const double2 *x, double m, double sc,
              double a) {
  const Geom &geo = g->l->g;
  const double h = 0.5 * sc;
  const double aa = a / h, bb = m / h;
  const int init = (aa == 0.0 && bb == 0.0) ? 0 : (aa == 0.0 ? 1 : 2);
  return dslash64(g, par, block(r, geo, par), block(x, geo, 1 - par), block(x, geo, par),
                  block((const double2 *)r, geo, par), aa, bb, h, +1, init);
}

int apply_D(qexstag_links_s *g, double2 *r, const double2 *x, double m, double sc) {
  int rc = stagD_par(g, 0, r, x, m, sc, 0.0);
  if (rc) return rc;
  return stagD_par(g, 1, r, x, m, sc, 0.0);
}

static int solve_xx_internal(qexstag_links_s *g, int par, double2 *y, const double2 *b, double m,
                             double r2req, int maxits, const qexstag_solver_params *p,
                             qexstag_solver_stats *st) {
  // solveXXInternal: y := 0 everywhere, then y_par from the inner solve
  const Geom &geo = g->l->g;
  int rc = vzero(VecD{y, geo.V}, geo.V);
  if (rc) return rc;
  return inner_solve(g, par, m, block(b, geo, par), block(y, geo, par), r2req, maxits, p, st);
}

static int recon_r(qexstag_links_s *g, double2 *x, const double2 *b, double m, double r2req,
                   int maxits, double b2e, double b2o, const qexstag_solver_params *p,
                   qexstag_solver_stats *st, double2 *y) {
  const Geom &geo = g->l->g;
  double b2 = b2e + b2o, r2stop = r2req * b2, r2stop2 = 0.5 * r2stop;
  double r2stope = (b2o <= r2stop2) ? r2stop - b2o : r2stop2;
  int rc;
  if (b2e > r2stope) {
    if ((rc = solve_xx_internal(g, 0, y, b, m, r2stope / b2e, maxits, p, st))) return rc;
    if ((rc = vscale(block(y, geo, 0), 4.0, geo.nh))) return rc;
    return apply_D(g, x, y, m, -1.0);
  }
  double r2stopo = (b2e <= r2stop2) ? r2stop - b2e : r2stop2;
  if (b2o > r2stopo) {
    if ((rc = solve_xx_internal(g, 1, y, b, m, r2stopo / b2o, maxits, p, st))) return rc;
    if ((rc = vscale(block(y, geo, 1), 4.0, geo.nh))) return rc;
    return apply_D(g, x, y, m, -1.0);
  }
  return QEXSTAG_OK;
}

static int recon_l(qexstag_links_s *g, double2 *x, const double2 *b, double m, double r2req,
                   int maxits, double b2e, double b2o, const qexstag_solver_params *p,
                   qexstag_solver_stats *st, double2 *d) {
  const Geom &geo = g->l->g;
  int rc;
  if ((rc = apply_D(g, d, b, m, -1.0))) return rc;  // d = Ddag b
  double d2e = 0;
  if ((rc = vnorm2(block((const double2 *)d, geo, 0), geo.nh, &d2e))) return rc;
  double req = 0.99 * r2req * (b2e + b2o) * m * m / d2e;
  if ((rc = solve_xx_internal(g, 0, x, d, m, req, maxits, p, st))) return rc;
  if ((rc = vscale(block(x, geo, 0), 4.0, geo.nh))) return rc;
  // eoReconstruct (stagD.nim:633-637): x_o = (b_o - D_oe x_e)/m
  if ((rc = stagD_par(g, 1, x, x, 0.0, -1.0 / m, 0.0))) return rc;
  return vaxpy(block(x, geo, 1), 1.0 / m, block(b, geo, 1), geo.nh);
}

int solve_full(qexstag_links_s *g, double2 *x, const double2 *b, double m,
               const qexstag_solver_params *p, qexstag_solver_stats *st) {
  const Geom &geo = g->l->g;
  const int V = geo.V, nh = geo.nh;
  Workspace &ws = g->ws;
  void *pr, *py, *pd;
  const size_t fb = sizeof(double2) * 3 * (size_t)V;
  int rc;
  if ((rc = ws.get(kSlotFull0, fb, &pr)) || (rc = ws.get(kSlotFull1, fb, &py)) ||
      (rc = ws.get(kSlotFull2, fb, &pd)))
    return rc;
  double2 *r = (double2 *)pr, *y = (double2 *)py, *d = (double2 *)pd;
  VecD xf{x, V}, rf{r, V};
  double b2 = 0;
  if ((rc = vnorm2(CVecD{b, V}, V, &b2))) return rc;
  if (!std::isfinite(b2)) return fail(QEXSTAG_ERR_NAN, "solve: source is not finite");
  double r2stop = p->r2req * b2;
  if (p->use_prev_soln) {
    if ((rc = apply_D(g, r, x, m, 1.0))) return rc;
    if ((rc = vsub(rf, CVecD{b, V}, cv(rf), V))) return rc;
  } else {
    if ((rc = vzero(xf, V))) return rc;
    if ((rc = vcopy(rf, CVecD{b, V}, V))) return rc;
  }
  double r2e = 0, r2o = 0;
  if ((rc = vnorm2(block((const double2 *)r, geo, 0), nh, &r2e))) return rc;
  if ((rc = vnorm2(block((const double2 *)r, geo, 1), nh, &r2o))) return rc;
  double r2 = r2e + r2o;
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  while (r2 > r2stop) {
    int mx = maxits - st->iterations;
    if (mx <= 0) break;
    double req = r2stop / r2;
    // solveInner (stagSolve.nim:313-326)
    double rb2 = r2e + r2o, rs = req * rb2, rs2 = 0.5 * rs;
    double rse = (r2o <= rs2) ? rs - r2o : rs2;
    double rso = (r2e <= rs2) ? rs - r2e : rs2;
    if ((rc = vzero(VecD{y, V}, V))) return rc;
    if (r2e <= rse || r2o <= rso || m == 0.0)
      rc = recon_r(g, y, r, m, req, mx, r2e, r2o, p, st, d);
    else
      rc = recon_l(g, y, r, m, req, mx, r2e, r2o, p, st, d);
    if (rc < 0) return rc;
    st->outer_iterations += 1;
    if ((rc = vaxpy(xf, 1.0, CVecD{y, V}, V))) return rc;
    if ((rc = apply_D(g, r, x, m, 1.0))) return rc;
    if ((rc = vsub(rf, CVecD{b, V}, cv(rf), V))) return rc;
    if ((rc = vnorm2(block((const double2 *)r, geo, 0), nh, &r2e))) return rc;
    if ((rc = vnorm2(block((const double2 *)r, geo, 1), nh, &r2o))) return rc;
    r2 = r2e + r2o;
    if (std::isnan(r2)) return fail(QEXSTAG_ERR_NAN, "solve: NaN residual");
  }
  st->r2 = b2 > 0 ? r2 / b2 : 0.0;
  return (r2 > r2stop) ? QEXSTAG_NOT_CONVERGED : QEXSTAG_OK;
}

}  // namespace qs
