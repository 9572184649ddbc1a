// phases.cu -- staggered phases and boundary signs on the device link copy.
// Multiplying by the signs twice restores the links, so the same call folds
// phases in and out.
//
// rephase_links(g, literal = true) is QEX's rephase exactly (setBC then
// stagPhase, src/physics/stagD.nim:106-114, 560-571,
// src/gauge/gaugeUtils.nim:133-140): both act on the first four fields of the
// operator's list, whatever its length -- field k gets eta_k(x) (phases
// [8,9,11,0]) and field 3 gets -1 on the last time slice.  For a naive list
// those are the four directions.  For newStag3's interleaved list
// [fat_0, long_0, fat_1, long_1, ...] QEX's call therefore phases fat_0,
// long_0, fat_1, long_1 with eta_0..eta_3, puts the boundary sign on long_1
// and leaves the rest unchanged; the literal form reproduces that.
//
// rephase_links(g, literal = false) phases every field of the list by its own
// direction and hop, which QEX has no single call for: one-hop links of
// direction mu get eta_mu(x) and -1 on the last time slice for mu = 3;
// three-hop long links get eta_mu(x) and -1 when the hop crosses the time
// boundary (the product of their three one-hop signs).
#include "lib.cuh"
#include "lowprec.cuh"

namespace qs {

int build_low_links(qexstag_links_s *g);
void free_low_links(LowLinks &low);

// NL fields of the list are rephased, field l as direction Hop<NL>::mu(l)
// with hop Hop<NL>::len(l) (NL = 4: fields 0-3 as directions 0-3, one hop)
template <int NL>
__global__ void rephase_kernel(Geom g, double2 *__restrict__ u) {
  const size_t V = (size_t)g.V;
  const int total = g.V * NL;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int l = t / g.V;
    const int site = t - l * g.V;
    const int par = site >= g.nh ? 1 : 0;
    int x[4], lex;
    site_coords(g, par, site - par * g.nh, x, lex);
    const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
    float s = eta_sign(mu, x);
    if (mu == 3 && x[3] + len >= g.L[3]) s = -s;
    if (s < 0.f) {
      double2 *ul = u + (size_t)l * 9 * V + site;
#pragma unroll
      for (int e = 0; e < 9; e++) {
        double2 v = ul[(size_t)e * V];
        ul[(size_t)e * V] = make_double2(-v.x, -v.y);
      }
    }
  }
}

int rephase_links(qexstag_links_s *g, bool literal) {
  const Geom &geo = g->l->g;
  const int grid = grid_for((long)geo.V * g->nl, kBlock, 8);
  if (g->nl == 8 && !literal)
    rephase_kernel<8><<<grid, kBlock, 0, stream()>>>(geo, g->u64);
  else
    rephase_kernel<4><<<grid, kBlock, 0, stream()>>>(geo, g->u64);
  note_launch();
  QS_LAUNCH_CHECK();
  free_low_links(g->low);
  return build_low_links(g);
}

}  // namespace qs
