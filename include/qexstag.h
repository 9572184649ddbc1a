/*
 * qexstag.h -- C ABI of the B200 (sm_100a) staggered-fermion library.
 *
 * This is the boundary a QEX (Nim) host calls through {.importc, dynlib.},
 * in the same way QEX already calls QUDA's MILC interface
 * (src/quda/quda_milc_interface.nim:289-295, called from
 * src/quda/qudaWrapperImpl.nim:252-255).  Every entry point takes plain C
 * types; none takes a C++ or torch type.
 *
 * Conventions
 *  - Every function returns an int status: QEXSTAG_OK (0); a positive value
 *    when a solver stopped without reaching its target (the result is still
 *    written); a negative QEXSTAG_ERR_* on error.  qexstag_last_error()
 *    returns a text description of the last error on the calling thread.
 *  - Lattice: dims[4] = {L0,L1,L2,L3}, each even and >= 4.  Sites are
 *    numbered as QEX numbers them with SIMD width 1 on one rank
 *    (src/layout/qlayout.nim:108-136):
 *      lex = x0 + L0*(x1 + L1*(x2 + L2*x3)),
 *      idx = (lex + (x0+x1+x2+x3 odd ? V : 0)) / 2,
 *    so even sites are [0, V/2) and odd sites [V/2, V).
 *  - Host fields (QEXSTAG_MEM_HOST) are in that order, array-of-structs:
 *      colour vector: double[V][3][2]              (re, im)
 *      link field k:  double[nlinks][V][3][3][2]   (row-major 3x3)
 *  - Device fields (QEXSTAG_MEM_DEVICE) are CUDA device pointers in the
 *    library's structure-of-arrays layout, which coalesces on the GPU:
 *      colour vector: double2[3][V]   (colour-major, then site index)
 *    Even-parity-only vectors may instead be given as double2[3][V/2]
 *    where an entry point says so.
 *  - Link lists follow QEX's Staggered.g: nlinks == 4 is naive staggered
 *    (link k = direction k, one hop); nlinks == 8 is fat+Naik interleaved as
 *    newStag3 builds it (src/physics/stagD.nim:40-51, 603-615): link 2*mu is
 *    the fat link (hop 1), link 2*mu+1 the long link (hop 3).  Links must
 *    already carry the staggered phases and boundary signs (QEX's
 *    setBC + stagPhase, src/physics/stagD.nim:106-114, 560-571).
 *  - Calls on one handle are not reentrant; separate handles and separate
 *    devices may be used from separate threads.  Work is issued on the
 *    stream set by qexstag_set_stream (default: the legacy default stream).
 */
#ifndef QEXSTAG_H
#define QEXSTAG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define QEXSTAG_OK 0
#define QEXSTAG_NOT_CONVERGED 1
#define QEXSTAG_ERR_ARG (-1)
#define QEXSTAG_ERR_CUDA (-2)
#define QEXSTAG_ERR_NAN (-3)
#define QEXSTAG_ERR_TIMEOUT (-4)
#define QEXSTAG_ERR_ALLOC (-5)
#define QEXSTAG_ERR_STATE (-6)
#define QEXSTAG_ERR_IO (-7)     /* gauge file: unreadable, malformed or failed checksum */

/* where field pointers live */
#define QEXSTAG_MEM_HOST 0
#define QEXSTAG_MEM_DEVICE 1

/* parities / subsets, as QEX's "even", "odd", "all" */
#define QEXSTAG_EVEN 0
#define QEXSTAG_ODD 1
#define QEXSTAG_ALL 2

/* inner-solver precision, QEX's SloppyType (src/solvers/solverBase.nim:8-9) */
#define QEXSTAG_SLOPPY_NONE 0
#define QEXSTAG_SLOPPY_SINGLE 1
#define QEXSTAG_SLOPPY_HALF 2

typedef struct qexstag_layout_s qexstag_layout;
typedef struct qexstag_links_s qexstag_links;

/* Solver inputs: the input half of QEX's SolverParams
   (src/solvers/solverBase.nim:10-17).  r2req is the squared relative
   residual, |b - A x|^2 <= r2req |b|^2 (src/solvers/cg.nim:155). */
typedef struct {
  double r2req;
  int maxits;
  int sloppy;          /* QEXSTAG_SLOPPY_* */
  double delta;        /* reliable-update threshold for sloppy solves
                          (0: 0.1 for SINGLE, 0.3 for HALF) */
  int verbosity;
  int use_prev_soln;   /* solve(): start from the x passed in */
  int reserved[6];
} qexstag_solver_params;

/* Solver outputs: the output half of QEX's SolverParams
   (src/solvers/solverBase.nim:18-28). */
typedef struct {
  int calls;
  int iterations;        /* Krylov iterations, all precisions */
  int outer_iterations;  /* defect-correction / refinement passes */
  int reliable_updates;
  double seconds;        /* device time of the call */
  double flops;          /* QEX's count, (nlinks*4*72+60)*nEven per iteration */
  double r2;             /* final true |b - A x|^2 / |b|^2 (FP64) */
  long long kernel_launches;  /* library kernels launched by the call */
} qexstag_solver_stats;

/* ---- runtime ---- */

/* Select the CUDA device for the calling thread and set the library up on
   it.  Replaces qexInit's device part; QUDA's initQuda analogue. */
int qexstag_init(int device);
/* Free every handle-independent resource on the current device. */
int qexstag_finalize(void);
/* Issue subsequent work on this cudaStream_t (NULL: legacy default). */
int qexstag_set_stream(void *stream);
/* Text of the last error on the calling thread (never NULL). */
const char *qexstag_last_error(void);
/* Block until all work issued by the library on its stream is done. */
int qexstag_synchronize(void);

/* ---- layout (src/layout/qlayout.nim, src/layout/shiftX.nim) ---- */

/* Build the V=1 checkerboard layout for dims (newLayout with SIMD width 1,
   src/layout/layoutX.nim:71-180). */
int qexstag_layout_create(const int dims[4], qexstag_layout **out);
int qexstag_layout_destroy(qexstag_layout *l);
/* Site index of coordinates x (qlayout.nim:108-136, layoutIndexQ). */
int qexstag_layout_index(const qexstag_layout *l, const int x[4], int64_t *idx);
/* Neighbour table of ShiftB(mu, len, subset) (src/layout/shifts.nim:18-44,
   src/layout/qshifts.nim:187-223): out_host[i] = index of x(i) + len*mu for
   each destination site i of the subset, in subset order.  Computed on the
   GPU with the index arithmetic the kernels use, then copied to host. */
int qexstag_layout_shift_table(const qexstag_layout *l, int mu, int len, int subset,
                               int32_t *out_host);

/* ---- links (Staggered.g, src/physics/stagD.nim:68-86, 573-615) ---- */

/* Upload a link list and build every precision the solvers use: FP64,
   FP32 and FP16 copies, and 12-real (two-row) long links when the long
   links are long_coeff times a phase times an SU(3) matrix to FP32 rounding
   (checked here; otherwise long links keep all 18 reals).  links points to
   nlinks*V*18 doubles in the host layout (mem == QEXSTAG_MEM_HOST) or to
   double2[nlinks][9][V] on the device (mem == QEXSTAG_MEM_DEVICE).  The
   handle keeps a pointer to l. */
int qexstag_links_create(qexstag_layout *l, int nlinks, const double *links, int mem,
                         double long_coeff, qexstag_links **out);
int qexstag_links_destroy(qexstag_links *g);
/* Replace the link data of a handle (same layout and nlinks) and rebuild its
   reduced-precision copies.  QEX's Staggered.g references the gauge fields,
   so an HMC update of U is seen by the next solve; with device copies the
   caller calls this after changing the links. */
int qexstag_links_update(qexstag_links *g, const double *links, int mem);
/* QEX's rephase(s) (src/physics/stagD.nim:106-114), literally: setBC
   (src/gauge/gaugeUtils.nim:133-140) negates field 3 of the list on the last
   time slice and stagPhase (stagD.nim:560-571) multiplies fields 0..3 by
   eta_0..eta_3 (phases [8,9,11,0]).  For a naive list these are the four
   directions.  For a fat+Naik list, as in QEX, only the first four fields
   [fat_0, long_0, fat_1, long_1] change (eta_0..eta_3, BC on long_1); use
   qexstag_links_rephase_all to phase every field by its own direction.
   Applying it twice restores the links; reduced copies are rebuilt. */
int qexstag_links_rephase(qexstag_links *g);
/* Every field of the list by its own direction and hop (no single QEX call
   does this): one-hop links of direction mu get eta_mu(x), and -1 on the
   last time slice for mu = 3; three-hop long links get eta_mu(x), and -1
   when the hop crosses the time boundary (the product of their three
   one-hop signs), as QEX's HISQ path folds them (stagPhase and setBC before
   smearing, src/hmc/hmcAction.nim:540-555).  Applying it twice restores the
   links; reduced copies are rebuilt. */
int qexstag_links_rephase_all(qexstag_links *g);
/* Links in MILC order, as QUDA's MILC interface takes them
   (QUDA_MILC_GAUGE_ORDER, which QEX's QUDA wrapper fills from Staggered.g at
   src/quda/qudaWrapperImpl.nim:134-139, 205-245): host arrays with the four
   directions of a site together, fat[V][4][3][3][2] and, for a fat+Naik
   operator, lng[V][4][3][3][2] (lng == NULL: a naive operator), sites in
   the V=1 order above, phases folded in.  The handle is the one
   qexstag_links_create makes from QEX's list [fat_0, long_0, ..., fat_3,
   long_3] (or [U_0 .. U_3]). */
int qexstag_links_create_milc(qexstag_layout *l, const double *fat, const double *lng, double long_coeff,
                              qexstag_links **out);
int qexstag_links_update_milc(qexstag_links *g, const double *fat, const double *lng);
/* Copy the handle's FP64 links out in MILC order (the inverse of
   qexstag_links_create_milc). */
int qexstag_links_get_milc(qexstag_links *g, double *fat, double *lng);
/* 1 when the handle uses 12-real long links in its reduced precisions. */
int qexstag_links_recon12(const qexstag_links *g);

/* ---- Dslash (src/physics/stagD.nim) ---- */

/* stagD2 (stagD.nim:383-448): on subset (EVEN or ODD)
     r = a*r + b*x + sum_k [U_k(s) x(s+d_k) - U_k(s-d_k)^dagger x(s-d_k)]. */
int qexstag_stagD2(qexstag_links *g, int subset, double *r, const double *x, double a,
                   double b, int mem);
/* stagDN (stagD.nim:451-455, the multi-vector sweep stagDPN 132-189): for
   i < n, on subset (EVEN or ODD)
     r[i] = m*x[i] + sum_k [U_k(s) x[i](s+d_k) - U_k(s-d_k)^dagger x[i](s-d_k)],
   which is stagD2(subset, r[i], x[i], 0, m) for n fields at once: each link
   is read once per site for up to 8 of them.  r and x hold n pointers to
   full-lattice fields; the other parity of each r[i] is not changed. */
int qexstag_stagDN(qexstag_links *g, int subset, int n, double *const *r, const double *const *x, double m,
                   int mem);
/* stagD (stagD.nim:459-462): r = a*r + m*x + (sc/2)(2D)x on subset
   (EVEN, ODD or ALL). */
int qexstag_stagD(qexstag_links *g, int subset, double *r, const double *x, double m,
                  double sc, double a, int mem);
/* D and Ddag (stagD.nim:617-622): r = m x +- (1/2)(2D) x on all sites. */
int qexstag_D(qexstag_links *g, double *r, const double *x, double m, int mem);
int qexstag_Ddag(qexstag_links *g, double *r, const double *x, double m, int mem);
/* stagD2ee / stagD2oo (stagD.nim:485-520): on one parity p,
   r_p = 4 m2 x_p - (2D)_pq (2D)_qp x_p.  Full-lattice fields. */
int qexstag_stagD2ee(qexstag_links *g, double *r, const double *x, double m2, int mem);
int qexstag_stagD2oo(qexstag_links *g, double *r, const double *x, double m2, int mem);
/* stagD2ee for device fields that allocates nothing; it has no counterpart in
   QEX.  For callers that cannot let a library call cudaMalloc: hosts whose
   own pool allocator already holds nearly all device memory, and hosts that
   cannot accept the device-wide synchronisation of cudaMalloc/cudaFree in
   the middle of an asynchronous pipeline.  r and x are device fields
   (double2[3][V]); the result equals qexstag_stagD2ee(..., MEM_DEVICE).  The
   odd-parity temporary is a static 3 MiB device array, so V/2 must be at most
   65536 (larger lattices return QEXSTAG_ERR_ARG); every GPU that loads the
   library holds it until exit.  All calls on a device share that array:
   calls that overlap on the GPU race.  The first call on a device looks up
   the array's address; make it before any stream capture.  The address is
   kept until qexstag_finalize; a host that resets the device calls
   qexstag_finalize before the reset (the module may load at another address
   afterwards), and the next call looks the address up again. */
int qexstag_stagD2ee_noalloc(qexstag_links *g, double *r, const double *x, double m2);

/* ---- solvers (src/physics/stagSolve.nim, src/solvers/cg.nim, cgm.nim) ---- */

/* solveEE / solveOO (stagSolve.nim:330-429): solve stagD2xx(m^2) r = x on
   the parity with FP64 defect correction around CG.  p->sloppy selects the
   inner precision (NONE: FP64 CG; SINGLE/HALF: FP32/FP16 reliable-update
   CG).  r is overwritten (QEX zeroes it). Full-lattice fields. */
int qexstag_solveEE(qexstag_links *g, double *r, const double *x, double m,
                    const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);
int qexstag_solveOO(qexstag_links *g, double *r, const double *x, double m,
                    const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);
/* solve (stagSolve.nim:469-557): D(m) x = b on the full lattice with
   even-odd preconditioning and reconstruction (solveInner). */
int qexstag_solve(qexstag_links *g, double *x, const double *b, double m,
                  const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);
/* Multi-mass solve (stagSolve.nim:560-668): D(ms[k]) xs[k] = b for
   k = 0..nmass-1 from multi-shift CG with shifts 4(ms[k]^2 - ms[0]^2). */
int qexstag_solve_multishift(qexstag_links *g, int nmass, double *const *xs,
                             const double *b, const double *ms,
                             const qexstag_solver_params *p, qexstag_solver_stats *st,
                             int mem);
/* Shifted systems on even sites for rational terms and several right-hand
   sides: (A + sigma[k]) y[j][k] = b[j], A = stagD2ee(m^2), for
   j < nrhs, k < nshift, with one multi-shift CG per batch of right-hand
   sides (links read once per site for all of them; cgm.nim:68-246), then,
   for p->sloppy != NONE, FP64 refinement of each (j,k) to p->r2req.
   b: nrhs pointers to full-lattice fields; y: nrhs*nshift pointers,
   y[j*nshift+k].  r2_out (optional): nrhs*nshift final true |res|^2/|b|^2. */
int qexstag_cgm_ee(qexstag_links *g, double m, int nshift, const double *sigma, int nrhs,
                   const double *const *b, double *const *y,
                   const qexstag_solver_params *p, qexstag_solver_stats *st,
                   double *r2_out, int mem);

/* Many independent even-site solves in one persistent launch: for each
   problem j (its own link handle, lattice and mass) solve
   stagD2ee(mass[j]^2) x[j] = b[j] on even sites as solveEE does (FP64 CG,
   cg.nim:55-272, then the FP64 true residual and defect correction,
   stagSolve.nim:330-421).  All problems iterate together in one cooperative
   kernel, captured in a CUDA graph; its block size and blocks per SM are
   chosen by timing candidates on the first call for a problem set.
   iterations[j] (and r2_out[j] = true |b - Ax|^2/|b|^2, optional) receive
   the per-problem results; launch_info (optional, 3 ints) receives the
   chosen block size, blocks per SM and 1 if the graph was used.  p->sloppy
   must be NONE; at most 128 problems, each with its own handle. */
int qexstag_solve_batched(int nprob, qexstag_links *const *g, const double *mass, double *const *x,
                          const double *const *b, const qexstag_solver_params *p, int *iterations,
                          double *r2_out, int *launch_info, qexstag_solver_stats *st, int mem);

/* ---- HMC force (src/hmc/hmcAction.nim:669-790, 851-885) ---- */

/* stagForceSolve followed by fermForce without smearing: solves
   stagD2ee(m^2) y = phi_e, psi = (4y, (2D)_oe 4y), then for every link k
   f_k(x) = projectTAH(s(x) psi(x) psi(x + d_k)^dagger U_k(x)^dagger),
   s = +1 on even and -1 on odd sites.  f: nlinks*V*18 doubles (host layout)
   or double2[nlinks][9][V] (device).  This is the f QEX passes to
   addForce(gf, 0.25*dtau, f). */
int qexstag_force(qexstag_links *g, double *f, const double *phi, double m,
                  const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);
/* fermForce alone for a given psi (full lattice). */
int qexstag_ferm_force(qexstag_links *g, double *f, const double *psi, int mem);
/* stagForceSolve (hmcAction.nim:669-721) alone: psi = (4y, (2D)_oe 4y) with
   stagD2ee(m^2) y = phi_e (full-lattice psi; the solve honours p->sloppy). */
int qexstag_force_solve(qexstag_links *g, double *psi, const double *phi, double m,
                        const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);
/* fermForce's outer products before the smearing chain rule and projection
   (hmcAction.nim:744-771): f_k(x) = s(x) psi(x) psi(x + d_k)^dagger, s = +1 on
   even and -1 on odd sites; for a fat+Naik list the long-link entries are
   QEX's f3.  These are what a smearing derivative (QEX's u.deriv(ff, f1, f3))
   consumes.  Layout as qexstag_force's f. */
int qexstag_ferm_outer(qexstag_links *g, double *f, const double *psi, int mem);

/* Self-test of the batched solver's grid barrier (the one wait inside a
   library kernel): a cooperative kernel of one block per SM passes the
   barrier twice, each wait limited to timeout_ms.  With missing = 0 it
   returns QEXSTAG_OK; with missing > 0 the barrier waits for that many
   blocks that never arrive, every block gives up after timeout_ms, and the
   call returns QEXSTAG_ERR_TIMEOUT with the device still usable. */
int qexstag_barrier_selftest(int missing, double timeout_ms);

/* ---- HISQ link smearing (src/gauge/fat7l.nim, src/physics/hisqLinks.nim,
   src/gauge/hisqsmear.nim) ----
   Gauge fields here are the four directions of a link field:
   double[4][V][3][3][2] on the host or double2[4][9][V] on the device, the
   layouts of qexstag_links_create with nlinks = 4.  QEX smears links with
   the staggered phases and boundary signs already folded in
   (hmcAction.nim:540-555 calls setBC and stagPhase before smearing). */

/* Fat7lCoefs (fat7l.nim:5-10) */
typedef struct {
  double one_link, three_staple, five_staple, seven_staple, lepage;
} qexstag_fat7_coefs;
/* HisqCoefs (hisqLinks.nim:3-8); reunit_eps is projectU's eps
   (matrixFunctions.nim:340-351, 1e-20) */
typedef struct {
  qexstag_fat7_coefs fat7first, fat7second;
  double naik;
  double reunit_eps;
} qexstag_hisq_coefs;
/* setHisqFat7 (hisqLinks.nim:10-15) */
void qexstag_fat7_coefs_set_hisq(qexstag_fat7_coefs *c, double f7lf, double naik);
/* newHISQ (hisqsmear.nim:53-64): first level (lepage, 0), second level
   (2 - lepage, naik), long-link coefficient -naik/24, reunit_eps 1e-20 */
void qexstag_hisq_coefs_init(qexstag_hisq_coefs *c, double lepage, double naik);

/* A smearing handle holds the device scratch of the staple sweeps (36 link
   fields of 144 B per site, plus staging); it keeps a pointer to l. */
typedef struct qexstag_smear_s qexstag_smear;
int qexstag_smear_create(qexstag_layout *l, qexstag_smear **out);
int qexstag_smear_destroy(qexstag_smear *s);
/* makeImpLinks (fat7l.nim:70-154): fl = fat7 smearing of gf with one-link,
   3-, 5-, 7-staple and Lepage terms; when naik != 0 and gf_long, ll are
   non-NULL also ll_mu(x) = naik gf_long_mu(x) gf_long_mu(x+mu)
   gf_long_mu(x+2mu). */
int qexstag_fat7(qexstag_smear *s, const qexstag_fat7_coefs *c, const double *gf, double *fl,
                 const double *gf_long, double *ll, double naik, int mem);
/* projectU (matrixFunctions.nim:340-351) of every link: u = x (x^dag x +
   eps)^(-1/2) */
int qexstag_project_u(qexstag_smear *s, const double *x, double *u, double eps, int mem);
/* HisqCoefs.smear (hisqLinks.nim:40-46): fat7 with fat7first, projectU, then
   fat7 with fat7second and the Naik product of the projected links. */
int qexstag_hisq_smear(qexstag_smear *s, const qexstag_hisq_coefs *c, const double *g, double *fat,
                       double *lng, int mem);
/* Smear thin links g into the fat+Naik handle (nlinks 8, same layout as s):
   its list becomes [fat_0, long_0, ..., fat_3, long_3] as newStag3 builds it
   from HISQ's outputs, and its reduced-precision copies are rebuilt.  The
   projected links are unitary, not special unitary, so the long links keep
   18 reals. */
int qexstag_links_hisq(qexstag_links *g, qexstag_smear *s, const qexstag_hisq_coefs *c, const double *thin,
                       int mem);

/* ---- chain rule through the smearing (src/gauge/fat7lderiv.nim,
   src/maths/matrixFunctions.nim:368-390, src/gauge/hisqsmear.nim:66-105) ----
   Derivatives follow QEX's convention: for a chain C on an output field and
   S = sum_x Re Tr C(x)^dagger out(x), the derivative with respect to an
   input field U is the field f with dS = sum_x Re Tr dU(x)^dagger f(x). */

/* fat7lDeriv (fat7lderiv.nim:122-331): deriv += derivative w.r.t. gauge of
   sum Re Tr mid^dag fat7(gauge); when naik != 0 and llgauge, llmid, llderiv
   are non-NULL also llderiv += derivative w.r.t. llgauge of
   sum Re Tr llmid^dag naik llgauge(x) llgauge(x+mu) llgauge(x+2mu).  Like
   QEX's, it adds to deriv and llderiv (which may be the same field when
   llgauge == gauge). */
int qexstag_fat7_deriv(qexstag_smear *s, const qexstag_fat7_coefs *c, const double *gauge, const double *mid,
                       double *deriv, const double *llgauge, const double *llmid, double *llderiv, double naik,
                       int mem);
/* projectUderiv (matrixFunctions.nim:368-390) of every link: r = derivative
   w.r.t. x of Re Tr chain^dag projectU(x), with u = projectU(x). */
int qexstag_project_u_deriv(qexstag_smear *s, const double *u, const double *x, const double *chain, double *r,
                            double eps, int mem);
/* smearGetForce's chain rule (hisqsmear.nim:66-105): deriv = derivative
   w.r.t. the thin links g of sum Re Tr (cfat^dag fat(g) + clong^dag long(g))
   for the smearing of qexstag_hisq_smear.  Recomputes the forward smearing
   of g.  cfat, clong are QEX's dsdsu, dsdsul (for the fermion force, its
   outer products f1 and f3). */
int qexstag_hisq_deriv(qexstag_smear *s, const qexstag_hisq_coefs *c, const double *g, const double *cfat,
                       const double *clong, double *deriv, int mem);
/* The staggered fermion force with HISQ smearing (QEX's force with
   StaggeredSmearing == "HISQ", hmcAction.nim:851-885 and fermForce
   723-790): smear the thin links into g (nlinks 8; its links are replaced),
   solve stagD2ee(m^2) y = phi_e (stagForceSolve), form the outer products
   f1, f3 of psi = (4y, (2D)_oe 4y) with the odd-site sign, take the chain
   rule through the smearing, and return f_mu = projectTAH(ff_mu U_mu^dag)
   on the thin links: the f QEX passes to addForce(gf, 0.25*dtau, f).  thin
   and f are 4-direction gauge fields, phi a full-lattice colour vector. */
int qexstag_hisq_force(qexstag_links *g, qexstag_smear *s, const qexstag_hisq_coefs *c, const double *thin,
                       double *f, const double *phi, double m, const qexstag_solver_params *p,
                       qexstag_solver_stats *st, int mem);

/* ---- gauge-field files (QEX's loadGauge / saveGauge,
   src/gauge/gaugeUtils.nim:96-131, over src/io/readerQiolite.nim and
   src/io/writerQiolite.nim; MILC files as src/new/milcIO.nim) ----
   The links are the 4-direction gauge field of qexstag_hisq_smear's
   convention (double[4][V][3][3][2] host, double2[4][9][V] device), without
   staggered phases, as QEX holds them between solves. */

#define QEXSTAG_GAUGE_SCIDAC 1  /* USQCD SciDAC single-file LIME (QIO layout), big-endian */
#define QEXSTAG_GAUGE_ILDG 2    /* ILDG LIME: SciDAC records plus ildg-format / ildg-binary-data */
#define QEXSTAG_GAUGE_MILC 3    /* MILC binary, version 5 (single precision) */

typedef struct {
  int format;                  /* QEXSTAG_GAUGE_* */
  int dims[4];
  int precision;               /* bytes per real in the file: 4 or 8 */
  int has_checksum;            /* the file stores a checksum */
  unsigned file_checksum[2];   /* as stored: SciDAC suma, sumb or MILC sum29, sum31 */
  unsigned data_checksum[2];   /* of the data read (qexstag_gauge_read only) */
  char date[64];
  char file_metadata[256];     /* user XML of the file (truncated) */
  char record_metadata[256];   /* user XML of the record (truncated) */
} qexstag_gauge_info;

/* Format, lattice, precision and metadata of a gauge file, without reading
   the links (getFileLattice, readerQiolite.nim:11-17). */
int qexstag_gauge_file_info(const char *path, qexstag_gauge_info *info);
/* Read a SciDAC, ILDG or MILC gauge file into links (reordered to the
   layout's site index, converted to FP64) and verify its checksum on the
   GPU.  The file lattice must equal the layout's.  Returns QEXSTAG_ERR_IO
   on a checksum mismatch, with the links written and both checksums in
   info (which may be NULL). */
int qexstag_gauge_read(qexstag_layout *l, const char *path, double *links, int mem, qexstag_gauge_info *info);
/* Write links as a SciDAC or ILDG file (precision 4 or 8 bytes, with the
   scidac-checksum record) or a MILC file (precision 4, this machine's byte
   order); file_md and record_md are the user XML of the file and the
   record (may be NULL). */
int qexstag_gauge_write(qexstag_layout *l, const char *path, const double *links, int mem, int format,
                        int precision, const char *file_md, const char *record_md);

/* ---- gauge action, gauge force and the molecular-dynamics updates
   (src/gauge/gaugeAction.nim, src/gauge/gaugeUtils.nim:419-459, 1466-1493,
   src/hmc/hmcAction.nim:248-304) ----
   Link fields and momenta are 4-direction fields as for
   qexstag_hisq_smear (host double[4][V][3][3][2], device double2[4][9][V]);
   the gauge links carry no staggered phases. */

/* GaugeActionCoeffs (gaugeAction.nim:14-19), plaquette and rectangle terms */
typedef struct {
  double plaq, rect;
} qexstag_gauge_coefs;
/* gaugeActRect (gaugeAction.nim:51-53): plaq = (1 - 8 c1) beta, rect = c1
   beta; c1 = -1/12 is tree-level Symanzik, -0.331 Iwasaki, -1.4088 DBW2,
   0 Wilson. */
void qexstag_gauge_coefs_rect(qexstag_gauge_coefs *c, double beta, double c1);
/* gaugeAction1 (gaugeAction.nim:487-571): -(1/3) (plaq sum_{x,mu>nu} Re Tr
   P_munu(x) + rect sum_{x,mu!=nu} Re Tr R_munu(x)). */
int qexstag_gauge_action(qexstag_layout *l, const qexstag_gauge_coefs *c, const double *u, int mem,
                         double *action);
/* gaugeForce (gaugeAction.nim:576-779): f_mu(x) = projectTAH(U_mu(x) C_mu(x)),
   C the plaq/3- and rect/3-weighted sums of the paths that close each
   plaquette and rectangle through U_mu(x); along U -> exp(t T) U the action
   changes at rate Re Tr[T^dag f]. */
int qexstag_gauge_force(qexstag_layout *l, const qexstag_gauge_coefs *c, const double *u, double *f, int mem);
/* axexpmuly(u, eps, p, u) (gaugeUtils.nim:452-459): u <- expAH(eps p) u with
   QEX's expAH (scaling, degree-12 Taylor, squaring; matexp.nim:316-346). */
int qexstag_link_update(qexstag_layout *l, double *u, const double *p, double eps, int mem);
/* p <- p + a f (mdv's p -= f with a = -1, hmcAction.nim:288-296). */
int qexstag_momenta_update(qexstag_layout *l, double *p, const double *f, double a, int mem);
/* p = randomTAH (randTah3, gaugeUtils.nim:1466-1493): Gaussian su(3)
   momenta from a counter-based generator (Philox-4x32-10), link k of the
   field drawing from (k, counter) under key seed, so a (seed, counter) pair
   reproduces the field on any device. */
int qexstag_momenta_heatbath(qexstag_layout *l, double *p, unsigned long long seed, unsigned long long counter,
                             int mem);
/* kineticAction (hmcAction.nim:248-255): 0.5 sum |p|^2 - 16 V. */
int qexstag_kinetic_action(qexstag_layout *l, const double *p, int mem, double *t);

/* ---- domain decomposition along t (QEX's rankGeom split with ShiftB
   boundary exchanges: src/layout/shifts.nim:76-103, 263-294,
   src/layout/qshifts.nim:23-177, src/comms/halo.nim) ----
   The global lattice is split into nranks slabs of T = L3/nranks time
   slices (T even, at least 6 for fat+Naik links and 4 for naive links);
   rank r holds slices [r T, (r+1) T).  A rank's fields are its slab in the
   V=1 order of the local lattice {L0, L1, L2, T} (qexstag_domain_local_dims):
   links double[nlinks][Vloc][3][3][2] (host) or double2[nlinks][9][Vloc]
   (device), phases folded in with global coordinates; colour vectors as
   elsewhere.  Calls take the set of domains the calling process holds
   (every rank in one process, or one rank per process); all processes make
   the same calls in the same order. */
typedef struct qexstag_domain_s qexstag_domain;
int qexstag_domain_create(const int global_dims[4], int nranks, int rank, int nlinks, qexstag_domain **out);
/* Split along t, then z (QEX's rankGeom over several directions): grid[0]
   ranks along z and grid[1] along t, rank = rz + grid[0] rt holding z rows
   [rz Z, (rz+1) Z) of slices [rt T, (rt+1) T), Z = L2/grid[0] and T as
   above (both even, at least 6 with Naik links and 4 without); its local
   lattice is {L0, L1, Z, T}.  Ghost rows in z are exchanged after the t
   ghosts, so the corners come from the diagonal neighbours; grid[0] = 1
   keeps z ghosts, exchanged with the rank itself. */
int qexstag_domain_create_zt(const int global_dims[4], const int grid[2], int rank, int nlinks,
                             qexstag_domain **out);
int qexstag_domain_destroy(qexstag_domain *d);
int qexstag_domain_local_dims(const qexstag_domain *d, int dims[4]);
/* All nranks domains in this process (rank order), on the current device:
   boundaries are exchanged by device-to-device copies. */
int qexstag_domain_connect_local(qexstag_domain *const *doms, int n);
/* One domain per process: boundaries by NCCL send/receive and sums by NCCL
   all-reduce over a communicator of nranks, from an id that rank 0 made
   with qexstag_nccl_unique_id and every rank received. */
int qexstag_nccl_unique_id(void *id128);
int qexstag_domain_connect_nccl(qexstag_domain *d, const void *id128);
/* A communicator supplied by the host, for one domain per process without
   NCCL: the shape of QEX's Comm object (src/comms/comms.nim:6-28: pushSend,
   pushRecv, waitSends/waitRecvs, allReduce over float64), e.g. MPI, QMP or
   a test harness.  For each exchange the library stages the boundary faces
   in host memory, posts both receives and both sends, then calls wait_all;
   buffers stay valid until wait_all returns.  A message goes to rank `rank`
   with tag 0 (travelling up in t: my top slices to the up neighbour's lower
   ghosts), 1 (down in t), 2 (up in z) or 3 (down in z); the receiver posts
   the same tag, and messages with one tag between one pair of ranks are
   matched in the order they are posted.  all_reduce_sum replaces x[0..n) by
   its sum over all ranks, the same value on every rank.  Each callback
   returns 0 on success; any other value makes the library call fail with
   QEXSTAG_ERR_STATE. */
typedef struct {
  void *ctx;
  int (*push_send)(void *ctx, int rank, int tag, const void *buf, size_t bytes);
  int (*push_recv)(void *ctx, int rank, int tag, void *buf, size_t bytes);
  int (*wait_all)(void *ctx);
  int (*all_reduce_sum)(void *ctx, double *x, int n);
} qexstag_host_comm;
/* One domain per process, connected through comm (copied; comm->ctx must
   stay valid while the domain is in use).  Every process makes the same
   calls in the same order, as for NCCL. */
int qexstag_domain_connect_host(qexstag_domain *d, const qexstag_host_comm *comm);
/* Set each domain's links (links[k] for doms[k]) and exchange their
   boundary slices. */
int qexstag_domain_links(qexstag_domain *const *doms, int n, const double *const *links, int mem);
/* 1 when the domain's reduced-precision long links are stored with 12
   reals (their signs rebuilt from global coordinates), 0 otherwise or
   before qexstag_domain_links. */
int qexstag_domain_recon12(const qexstag_domain *d);
/* stagD2ee on the decomposed lattice: r[k] even sites from x[k]. */
int qexstag_domain_stagD2ee(qexstag_domain *const *doms, int n, double *const *r, const double *const *x, double m2,
                            int mem);
/* FP64 CG (cg.nim:55-272) for stagD2ee(m^2) y = b_e on the decomposed
   lattice, zero start: x[k] receives y on even sites and zeros on odd
   sites; st->r2 is the true relative residual over the whole lattice. */
int qexstag_domain_solveEE(qexstag_domain *const *doms, int n, double *const *x, const double *const *b, double m,
                           const qexstag_solver_params *p, qexstag_solver_stats *st, int mem);

/* ---- benchmark hook (QEX's src/bench/benchStagProp.nim times the operator
   the same way, host timers around repeated calls) ---- */

/* Time the even-parity Schur operator (two Dslash half sweeps) in precision
   prec (0 FP64, 1 FP32, 2 FP16 with the handle's reduced-precision links) on
   internal device vectors: seconds per call, averaged over nrep calls after
   two warm-up calls, from CUDA events on the library's stream. */
int qexstag_bench_schur(qexstag_links *g, int prec, int nrep, double m2,
                        double *seconds_per_call);

#ifdef __cplusplus
}
#endif
#endif /* QEXSTAG_H */
