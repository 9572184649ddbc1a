// mrhs.cu -- QEX's multi-right-hand-side Dslash in FP64 (stagDN over
// stagDPN, src/physics/stagD.nim:132-189, 451-455): for n colour vectors at
// once, on one parity,
//   r_i = m x_i + sum_k [U_k(s) x_i(s + d_k) - U_k(s - d_k)^dagger x_i(s - d_k)].
// QEX tiles 16 sites x 8 vectors so that a site's links are loaded once for
// all vectors.  Here a block of 256 threads is G warp-uniform groups of
// 256/G sites (G = 1, 2 or 4); group q applies the operator to vectors
// 2q and 2q+1 of its sites.  Every group reads the same links, so each link
// comes from HBM once per site and from L1 for the other groups, and every
// vector's loads stay coalesced across the warp.  Up to 8 vectors per
// launch.  Accumulation follows stagDPN: the mass term, then the forward
// hops, then the backward hops.
//
// Compulsory bytes per output site: links (nlinks x 2 x 144 B: a forward
// link at the site and a backward link at the neighbour) + n x (48 B own
// site, 48 B neighbours (L2-resident), 48 B out) -> fat+Naik, n = 8:
// 2304 + 1152 = 3456 B, against 8 x 2448 B for eight single-vector sweeps.
#include <algorithm>

#include "lib.cuh"

namespace qs {

constexpr int kDnPer = 2;  // vectors per thread
constexpr int kDnMax = 8;  // vectors per launch

struct DnArgs {
  Geom g;
  const double2 *u;       // double2 [nlinks][9][V]
  int po;                 // output parity
  int n;                  // vectors in this launch
  int groups;             // G: threads of a block per site
  double m;
  const double2 *x[kDnMax];  // full-lattice fields, double2 [3][xstride]
  double2 *r[kDnMax];
  int xstride, rstride;
};

template <int NL>
__global__ void __launch_bounds__(kBlock, 2) dslashN64_kernel(const DnArgs A) {
  const Geom &g = A.g;
  const int nh = g.nh;
  const size_t V = (size_t)g.V;
  const int S = blockDim.x / A.groups;  // sites per block step
  const int grp = threadIdx.x / S, sl = threadIdx.x - grp * S;
  const int j0 = grp * kDnPer;
  if (j0 >= A.n) return;
  const int nq = min(kDnPer, A.n - j0);
  const size_t in_base = (size_t)(1 - A.po) * nh, out_base = (size_t)A.po * nh;
  for (int k = blockIdx.x * S + sl; k < nh; k += gridDim.x * S) {
    int x[4], lex;
    site_coords(g, A.po, k, x, lex);
    double2 acc[kDnPer][3];
#pragma unroll
    for (int q = 0; q < kDnPer; q++) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        double2 v = make_double2(0.0, 0.0);
        if (q < nq) v = ldg(A.x[j0 + q] + (size_t)c * A.xstride + out_base + k);
        acc[q][c] = make_double2(A.m * v.x, A.m * v.y);
      }
    }
    // forward hops: + U_l(s) x(s + d_l)
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const int jf = nbr_half(g, x, lex, mu, len);
      const double2 *ul = A.u + (size_t)l * 9 * V + out_base + k;
      double2 u[9];
#pragma unroll
      for (int e = 0; e < 9; e++) u[e] = ldlink(ul + (size_t)e * V);
#pragma unroll
      for (int q = 0; q < kDnPer; q++) {
        if (q < nq) {
          const double2 *xq = A.x[j0 + q] + in_base + jf;
          double2 v[3];
#pragma unroll
          for (int c = 0; c < 3; c++) v[c] = ldg(xq + (size_t)c * A.xstride);
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int c = 0; c < 3; c++) acc[q][i] = cmadd(acc[q][i], u[3 * i + c], v[c]);
        }
      }
    }
    // backward hops: - U_l(s - d_l)^dagger x(s - d_l)
#pragma unroll
    for (int l = 0; l < NL; l++) {
      const int mu = Hop<NL>::mu(l), len = Hop<NL>::len(l);
      const int jb = nbr_half(g, x, lex, mu, -len);
      const double2 *ul = A.u + (size_t)l * 9 * V + in_base + jb;
      double2 u[9];
#pragma unroll
      for (int e = 0; e < 9; e++) u[e] = ldlink(ul + (size_t)e * V);
#pragma unroll
      for (int q = 0; q < kDnPer; q++) {
        if (q < nq) {
          const double2 *xq = A.x[j0 + q] + in_base + jb;
          double2 w[3];
#pragma unroll
          for (int c = 0; c < 3; c++) w[c] = ldg(xq + (size_t)c * A.xstride);
#pragma unroll
          for (int i = 0; i < 3; i++) {
            double2 t = make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < 3; c++) t = cjmadd(t, u[3 * c + i], w[c]);
            acc[q][i].x -= t.x;
            acc[q][i].y -= t.y;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kDnPer; q++) {
      if (q < nq) {
        double2 *rq = A.r[j0 + q] + out_base + k;
#pragma unroll
        for (int c = 0; c < 3; c++) rq[(size_t)c * A.rstride] = acc[q][c];
      }
    }
  }
}

// r[i] (parity po) = m x[i] + (2D) x[i] for i < n; full-lattice device
// fields with strides xstride, rstride.  Vectors go 8 to a launch.
int dslashN64(const qexstag_links_s *gl, int po, int n, double2 *const *r, int rstride, const double2 *const *x,
              int xstride, double m) {
  const Geom &g = gl->l->g;
  for (int i0 = 0; i0 < n; i0 += kDnMax) {
    DnArgs A;
    A.g = g;
    A.u = gl->u64;
    A.po = po;
    A.n = std::min(kDnMax, n - i0);
    A.groups = A.n <= 2 ? 1 : (A.n <= 4 ? 2 : 4);
    A.m = m;
    for (int j = 0; j < kDnMax; j++) {
      A.x[j] = j < A.n ? x[i0 + j] : nullptr;
      A.r[j] = j < A.n ? r[i0 + j] : nullptr;
    }
    A.xstride = xstride;
    A.rstride = rstride;
    const int S = kBlock / A.groups;
    const int grid = (int)std::min<long>(((long)g.nh + S - 1) / S, (long)num_sms() * 4);
    if (gl->nl == 8)
      dslashN64_kernel<8><<<grid, kBlock, 0, stream()>>>(A);
    else
      dslashN64_kernel<4><<<grid, kBlock, 0, stream()>>>(A);
    note_launch();
    QS_LAUNCH_CHECK();
  }
  return QEXSTAG_OK;
}

}  // namespace qs
