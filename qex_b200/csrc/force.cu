// force.cu -- staggered fermion force without smearing (QEX fermForce,
// src/hmc/hmcAction.nim:723-790, with the identity chain rule):
//   f1_k(x) = s(x) psi(x) psi(x + d_k)^dagger   (s = +1 even, -1 odd sites)
//   f_k(x)  = projectTAH(f1_k(x) U_k(x)^dagger)   (matrixFunctions.nim:414-419)
// for every link k of the list (fat hops d = mu, long hops d = 3 mu).
// One thread per site and link; psi(x) and psi(x+d) are gathered from the
// full-lattice field, U and f streamed as 16-byte words.
#include "lib.cuh"

namespace qs {

template <int NL>
__global__ void __launch_bounds__(kBlock)
    ferm_force_kernel(Geom g, const double2 *__restrict__ u, const double2 *__restrict__ psi,
                      double2 *__restrict__ f) {
  const size_t V = (size_t)g.V;
  const int total = g.V * NL;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int l = t / g.V;
    const int site = t - l * g.V;
    const int par = site >= g.nh ? 1 : 0;
    const int k = site - par * g.nh;
    int x[4], lex;
    site_coords(g, par, k, x, lex);
    const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
    const size_t nb = (size_t)(1 - par) * g.nh + nbr_half(g, x, lex, mu, len);
    double2 a[3], b[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      a[c] = ldg(psi + (size_t)c * V + site);
      b[c] = ldg(psi + (size_t)c * V + nb);
    }
    const double s = par ? -1.0 : 1.0;
    const double2 *ul = u + (size_t)l * 9 * V + site;
    double2 um[9];
#pragma unroll
    for (int e = 0; e < 9; e++) um[e] = ldlink(ul + (size_t)e * V);
    // w_j = sum_q conj(b_q) conj(U_{jq}) = conj((U b)_j);  m_{pj} = s a_p w_j
    double2 w[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 ub = make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < 3; q++) ub = cmadd(ub, um[3 * j + q], b[q]);
      w[j] = make_double2(s * ub.x, -s * ub.y);
    }
    double2 m[9];
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        double2 ap = a[p], wj = w[j];
        m[3 * p + j] = make_double2(ap.x * wj.x - ap.y * wj.y, ap.x * wj.y + ap.y * wj.x);
      }
    // projectTAH: (m - m^dagger)/2 minus the trace part
    double2 r[9];
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        double2 mpj = m[3 * p + j], mjp = m[3 * j + p];
        r[3 * p + j] = make_double2(0.5 * (mpj.x - mjp.x), 0.5 * (mpj.y + mjp.y));
      }
    const double tr = (r[0].y + r[4].y + r[8].y) * (1.0 / 3.0);
    r[0].y -= tr;
    r[4].y -= tr;
    r[8].y -= tr;
    double2 *fl = f + (size_t)l * 9 * V + site;
#pragma unroll
    for (int e = 0; e < 9; e++) __stcs(fl + (size_t)e * V, r[e]);
  }
}

// fermForce's outer products alone (hmcAction.nim:744-771), before the
// smearing chain rule and the projection: f_k(x) = s(x) psi(x) psi(x+d_k)^dagger
template <int NL>
__global__ void __launch_bounds__(kBlock)
    ferm_outer_kernel(Geom g, const double2 *__restrict__ psi, double2 *__restrict__ f) {
  const size_t V = (size_t)g.V;
  const int total = g.V * NL;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int l = t / g.V;
    const int site = t - l * g.V;
    const int par = site >= g.nh ? 1 : 0;
    int x[4], lex;
    site_coords(g, par, site - par * g.nh, x, lex);
    const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
    const size_t nb = (size_t)(1 - par) * g.nh + nbr_half(g, x, lex, mu, len);
    double2 a[3], b[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      a[c] = ldg(psi + (size_t)c * V + site);
      b[c] = ldg(psi + (size_t)c * V + nb);
    }
    const double s = par ? -1.0 : 1.0;
    double2 *fl = f + (size_t)l * 9 * V + site;
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const double2 ap = a[p], bq = b[q];
        // s * a_p * conj(b_q)
        __stcs(fl + (size_t)(3 * p + q) * V,
               make_double2(s * (ap.x * bq.x + ap.y * bq.y), s * (ap.y * bq.x - ap.x * bq.y)));
      }
  }
}

int ferm_outer64(qexstag_links_s *g, double2 *f, const double2 *psi) {
  const Geom &geo = g->l->g;
  const int grid = grid_for((long)geo.V * g->nl, kBlock, 8);
  if (g->nl == 8)
    ferm_outer_kernel<8><<<grid, kBlock, 0, stream()>>>(geo, psi, f);
  else
    ferm_outer_kernel<4><<<grid, kBlock, 0, stream()>>>(geo, psi, f);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

int ferm_force64(qexstag_links_s *g, double2 *f, const double2 *psi) {
  const Geom &geo = g->l->g;
  const long total = (long)geo.V * g->nl;
  const int grid = grid_for(total, kBlock, 8);
  if (g->nl == 8)
    ferm_force_kernel<8><<<grid, kBlock, 0, stream()>>>(geo, g->u64, psi, f);
  else
    ferm_force_kernel<4><<<grid, kBlock, 0, stream()>>>(geo, g->u64, psi, f);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

}  // namespace qs
