// mixed.cu -- reduced-precision link copies, the sloppy (FP32 / FP16)
// reliable-update CG and the multi-shift solvers.
#include "lib.cuh"

namespace qs {

int build_low_links(qexstag_links_s *g) {
  g->low = LowLinks();
  g->low.nfat = g->nl == 8 ? 4 : 4;
  g->low.nlong = g->nl == 8 ? 4 : 0;
  g->low.long_coeff = g->long_coeff;
  return QEXSTAG_OK;
}

void free_low_links(LowLinks &low) {
  cudaFree(low.f32_fat);
  cudaFree(low.f32_fat_tail);
  cudaFree(low.f32_long);
  cudaFree(low.f32_long_tail);
  cudaFree(low.f16_fat);
  cudaFree(low.f16_fat_tail);
  cudaFree(low.f16_long);
  cudaFree(low.f16_long_tail2);
  cudaFree(low.f16_long_tail);
  low = LowLinks();
}

int cg_mixed(qexstag_links_s *g, int par, double m2, CVecD b, VecD x, double r2req, int maxits,
             int sloppy, double delta, CgOut *out, int *reliable) {
  return fail(QEXSTAG_ERR_ARG, "sloppy solves are not available in this build");
}

int cgm_ee(qexstag_links_s *g, double m, int nshift, const double *sigma, int nrhs,
           const double2 *const *b, double2 *const *y, const qexstag_solver_params *p,
           qexstag_solver_stats *st, double *r2_out) {
  return fail(QEXSTAG_ERR_ARG, "cgm_ee is not available in this build");
}

int solve_multishift(qexstag_links_s *g, int nmass, double2 *const *xs, const double2 *b,
                     const double *ms, const qexstag_solver_params *p, qexstag_solver_stats *st) {
  return fail(QEXSTAG_ERR_ARG, "solve_multishift is not available in this build");
}

}  // namespace qs
