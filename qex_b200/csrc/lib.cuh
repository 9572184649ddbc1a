// lib.cuh -- host-side declarations shared between the library's
// translation units: the link handle, its device workspace and the kernel
// launchers.
#pragma once
#include <map>
#include <vector>

#include "internal.cuh"
#include "mixed.cuh"

namespace qs {

int runtime_ready();

// Device workspace owned by a link handle: buffers identified by a slot
// number, grown on demand, freed with the handle.
struct Workspace {
  std::map<int, std::pair<size_t, void *>> bufs;
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  int get(int slot, size_t bytes, void **out);
  int get_pinned(size_t bytes, void **out);
  void release();
};

// workspace slots
enum Slot {
  kSlotIn0 = 0,   // staged host input fields (SoA)
  kSlotIn1,
  kSlotOut0,      // staged outputs (SoA)
  kSlotOut1,
  kSlotAos,       // AoS staging for host transfers
  kSlotTmpOdd,    // stagD2xx temporary (other parity block)
  kSlotCgR, kSlotCgP, kSlotCgAp, kSlotCgT, kSlotCgX,
  kSlotCgState,
  kSlotDcRho, kSlotDcY, kSlotDcB,  // defect correction
  kSlotFull0, kSlotFull1, kSlotFull2,
  kSlotMx0 = 40,  // mixed-precision vectors and multishift (up to 80 slots)
  kSlotMs0 = 120,
  kSlotDn0 = 300,  // stagDN host staging: 8 inputs, then 8 outputs
  kSlotLast = 400
};

}  // namespace qs

struct qexstag_links_s {
  qexstag_layout_s *l = nullptr;
  int nl = 0;
  double long_coeff = 1.0;
  double2 *u64 = nullptr;  // [nl][9][V]
  qs::LowLinks low;        // FP32 / FP16 copies (mixed.cuh)
  qs::Workspace ws;
};

namespace qs {

// a colour-vector view: SoA double2 [3][stride], sites indexed from 0
struct VecD {
  double2 *p;
  int stride;
};
struct CVecD {
  const double2 *p;
  int stride;
};
inline CVecD cv(VecD v) { return CVecD{v.p, v.stride}; }
// parity block of a full-lattice field
inline VecD block(double2 *full, const Geom &g, int par) { return VecD{full + (size_t)par * g.nh, g.V}; }
inline CVecD block(const double2 *full, const Geom &g, int par) {
  return CVecD{full + (size_t)par * g.nh, g.V};
}

// ---- dslash.cu ----
// out = c*(a*rin + b*xs + hop*sum_k [...]) on the output parity po, with
// input field xin on the other parity and xs, rin on parity po.
// init: 0 -> zero, 1 -> b*xs, 2 -> a*rin + b*xs.
enum RedKind { kRedNone = 0, kRedCgPAp = 1, kRedDot = 2 };
int dslash64(const qexstag_links_s *g, int po, VecD out, CVecD xin, CVecD xs, CVecD rin,
             double a, double b, double c, int hop, int init, int red = kRedNone,
             void *state = nullptr, const int *done = nullptr, double *dot_out = nullptr);
// One domain of a decomposed lattice for the mixed-precision CG
// (mixed.cu: cg_mixed_domain): the links of its extended lattice, its
// interior even sites [even_lo, even_lo + n) and the odd sites
// [odd_lo, odd_hi) half sweep 1 must produce, and the decomposition's
// operations: the ghost exchange of an even field of 16-byte sites, the
// in-place sum over processes of one device double, and the FP64 Schur
// operator on compact interior fields (double2 [3][n]).
struct MxDomain {
  void *ctx;
  int (*exchange_even)(void *ctx, void *field);
  int (*allreduce)(void *ctx, double *dev, int n);  // n device doubles summed over the processes, in place
  int (*schur64)(void *ctx, const double2 *x, double2 *ax);
  qexstag_links_s *g;
  int even_lo, n, odd_lo, odd_hi;
};
struct CgOut;
int cg_mixed_domain(const MxDomain &D, double m2, const double2 *b, double2 *x, double r2req, int maxits,
                    double delta, CgOut *out, int *reliable);
// stagDN (mrhs.cu): r[i] (parity po) = m x[i] + (2D) x[i], i < n
int dslashN64(const qexstag_links_s *gl, int po, int n, double2 *const *r, int rstride, const double2 *const *x,
              int xstride, double m);
// Schur operator on parity par: r = 4 m2 x - (2D)_{par,q} (2D)_{q,par} x,
// with t (q block) the temporary; red kRedCgPAp/kRedDot accumulate Re<x, r>.
int schur64(const qexstag_links_s *g, int par, VecD r, CVecD x, VecD t, double m2,
            int red = kRedNone, void *state = nullptr, const int *done = nullptr,
            double *dot_out = nullptr);
int dslash64_ranges(const qexstag_links_s *gl, int po, VecD out, CVecD xin, CVecD xs, double b, double c,
                    int hop, int k0, int k1, int k2, int k3, const int *done);
int dslash64_rows(const qexstag_links_s *gl, int po, VecD out, CVecD xin, CVecD xs, double b, double c, int hop,
                  int k0, int nrun, int rowlen, int pitch, const int *done);

// ---- blas.cu ----
int aos_to_soa(const double *aos, double2 *soa, int n, int stride, int ncomp);
int soa_to_aos(const double2 *soa, double *aos, int n, int stride, int ncomp);
int vcopy(VecD y, CVecD x, int n);
int vzero(VecD y, int n);
int vscale(VecD y, double s, int n);
int vaxpy(VecD y, double a, CVecD x, int n);         // y += a x
int vxpay(VecD y, CVecD x, double a, int n);         // y = x + a y
int vaxpby(VecD y, double a, CVecD x, double b, int n);  // y = a x + b y
int vsub(VecD y, CVecD a, CVecD b, int n);           // y = a - b
// reductions to a device double (result) and, when host != nullptr, to host
int vnorm2(CVecD x, int n, double *host);
int vredot(CVecD x, CVecD y, int n, double *host);
// |a - b|^2 (no write)
int vdiffnorm2(CVecD a, CVecD b, int n, double *host);

// ---- solvers (cg.cu) ----
// Asynchronous read of a solver's device state: start() queues a copy into
// the pinned staging buffer and records an event; wait() blocks on that
// event only, so work queued after start() keeps the GPU busy meanwhile.
struct StateSnapshot {
  cudaEvent_t ev = nullptr;
  StateSnapshot() = default;
  StateSnapshot(const StateSnapshot &) = delete;
  StateSnapshot &operator=(const StateSnapshot &) = delete;
  ~StateSnapshot();
  int start(const void *dev, size_t bytes);
  int wait(void *host, size_t bytes);
};
struct CgOut {
  int iterations;
  double r2;  // recursive |r|^2/|b|^2 at exit
  int nan;
};
// FP64 CG (cg.nim, cpNone) on parity par for stagD2xx(m2) x = b, x zeroed.
int cg64(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits,
         CgOut *out);
// solveXX (stagSolve.nim:330-421): defect correction with inner solver of
// precision sloppy; r, x full-lattice device fields.
int solve_xx(qexstag_links_s *g, int par, double2 *r, const double2 *x, double m,
             const qexstag_solver_params *p, qexstag_solver_stats *st);
int solve_full(qexstag_links_s *g, double2 *x, const double2 *b, double m,
               const qexstag_solver_params *p, qexstag_solver_stats *st);

// ---- force.cu ----
int ferm_force64(qexstag_links_s *g, double2 *f, const double2 *psi);
int ferm_outer64(qexstag_links_s *g, double2 *f, const double2 *psi);

}  // namespace qs
