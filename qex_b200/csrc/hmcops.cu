// hmcops.cu -- the gauge and momentum side of an HMC step on the device:
//  - gauge action (gaugeAction1, src/gauge/gaugeAction.nim:487-571) and
//    gauge force (gaugeForce = gaugeActionDeriv + contractProjectTAH,
//    gaugeAction.nim:576-779, src/gauge/gaugeUtils.nim:419-441) for
//    plaquette + rectangle (Symanzik / Iwasaki / DBW2) coefficients;
//  - link update U <- expAH(eps P) U (axexpmuly, gaugeUtils.nim:452-459;
//    expAH, src/maths/matexp.nim:316-346);
//  - momentum update P += a F and refresh P = randomTAH (randTah3,
//    gaugeUtils.nim:1466-1493) from a counter-based generator;
//  - kinetic energy 0.5 |P|^2 - 16 V (kineticAction,
//    src/hmc/hmcAction.nim:248-255).
// Fields are 4-direction link fields double2[4][9][V] (the library's link
// layout).  The force gathers, per (site, direction), every plaquette and
// 2x1 rectangle through the link as the product of its other links, with the
// direction/parity-interleaved block order of the smearing sweeps.
#include <algorithm>

#include "smear.cuh"

namespace qs {

// t = t (F or F^dag) at site s; F streamed a row (or column) at a time
__device__ __forceinline__ void mul_link(M3 &t, const double2 *F, size_t V, int s, bool dag) {
  M3 r;
#pragma unroll
  for (int e = 0; e < 9; e++) r.e[e] = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double2 f[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      // (F^dag)_kj = conj(F_jk)
      const double2 v = __ldg(F + (size_t)(dag ? 3 * j + k : 3 * k + j) * V + s);
      f[j] = dag ? make_double2(v.x, -v.y) : v;
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) r.e[3 * i + j] = cmadd(r.e[3 * i + j], t.e[3 * i + k], f[j]);
  }
  t = r;
}
__device__ __forceinline__ void set_link(M3 &t, const double2 *F, size_t V, int s, bool dag) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double2 v = __ldg(F + (size_t)(dag ? 3 * j + i : 3 * i + j) * V + s);
      t.e[3 * i + j] = dag ? make_double2(v.x, -v.y) : v;
    }
}

struct PathCtx {
  const Geom *g;
  const SiteCtx *c;
  const double2 *u;
  int mu, nu;
};
// site x + a mu + b nu
__device__ __forceinline__ int at(const PathCtx &p, int a, int b) {
  if (b == 0) return a == 0 ? p.c->site : disp1(*p.g, p.c->x, p.c->lex, p.c->par, p.mu, a);
  if (a == 0) return disp1(*p.g, p.c->x, p.c->lex, p.c->par, p.nu, b);
  return disp2(*p.g, p.c->x, p.c->lex, p.c->par, p.mu, a, p.nu, b);
}
// one step of an open path: along +-nu from (a, b), or -mu from (a, b)
__device__ __forceinline__ void step_nu(M3 &t, const PathCtx &p, int a, int b, int s, bool first) {
  const size_t V = (size_t)p.g->V;
  const double2 *Un = p.u + (size_t)p.nu * 9 * V;
  const int site = s > 0 ? at(p, a, b) : at(p, a, b - 1);
  if (first)
    set_link(t, Un, V, site, s < 0);
  else
    mul_link(t, Un, V, site, s < 0);
}
__device__ __forceinline__ void step_back_mu(M3 &t, const PathCtx &p, int a, int b) {
  const size_t V = (size_t)p.g->V;
  mul_link(t, p.u + (size_t)p.mu * 9 * V, V, at(p, a - 1, b), true);
}

// acc += cp * (plaquette closers) + cr * (rectangle closers) of U_mu(x):
// open paths from x+mu back to x (Re Tr[U_mu(x) C] is the loop)
__device__ __forceinline__ void closers(M3 &acc, const Geom &g, const SiteCtx &c, const double2 *u, int mu,
                                        double cp, double cr) {
  const size_t V = (size_t)g.V;
#pragma unroll 1
  for (int k = 0; k < 3; k++) {
    PathCtx p{&g, &c, u, mu, other_dir(mu, k)};
#pragma unroll 1
    for (int s = -1; s <= 1; s += 2) {
      M3 t;
      // plaquette: x+mu -> x+mu+s nu -> x+s nu -> x
      step_nu(t, p, 1, 0, s, true);
      step_back_mu(t, p, 1, s);
      step_nu(t, p, 0, s, -s, false);
      m_axpy(acc, cp, t);
      if (cr == 0.0) continue;
      // long in mu, U_mu(x) first: x+mu -> x+2mu -> +s nu -> back 2 mu -> x
      set_link(t, u + (size_t)mu * 9 * V, V, at(p, 1, 0), false);
      step_nu(t, p, 2, 0, s, false);
      step_back_mu(t, p, 2, s);
      step_back_mu(t, p, 1, s);
      step_nu(t, p, 0, s, -s, false);
      m_axpy(acc, cr, t);
      // long in mu, U_mu(x) second: x+mu -> +s nu -> back 2 mu -> x-mu -> x
      step_nu(t, p, 1, 0, s, true);
      step_back_mu(t, p, 1, s);
      step_back_mu(t, p, 0, s);
      step_nu(t, p, -1, s, -s, false);
      mul_link(t, u + (size_t)mu * 9 * V, V, at(p, -1, 0), false);
      m_axpy(acc, cr, t);
      // long in nu: x+mu -> x+mu+2s nu -> x+2s nu -> x
      step_nu(t, p, 1, 0, s, true);
      step_nu(t, p, 1, s, s, false);
      step_back_mu(t, p, 1, 2 * s);
      step_nu(t, p, 0, 2 * s, -s, false);
      step_nu(t, p, 0, s, -s, false);
      m_axpy(acc, cr, t);
    }
  }
}

__device__ __forceinline__ void tah(M3 &r, const M3 &m) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double2 a = m.e[3 * i + j], b = m.e[3 * j + i];
      r.e[3 * i + j] = make_double2(0.5 * (a.x - b.x), 0.5 * (a.y + b.y));
    }
  const double t = (r.e[0].y + r.e[4].y + r.e[8].y) * (1.0 / 3.0);
  r.e[0].y -= t;
  r.e[4].y -= t;
  r.e[8].y -= t;
}

// F_mu(x) = projectTAH(U_mu(x) (cp sum P + cr sum R)), cp = plaq/3, cr = rect/3
__global__ void __launch_bounds__(kSmBlock) gauge_force_kernel(Geom g, const double2 *__restrict__ u, double2 *f,
                                                               double cp, double cr) {
  SiteCtx c;
  if (!site_of_thread(g, c)) return;
  const int mu = c.mu;
  const size_t V = (size_t)g.V;
  M3 acc;
#pragma unroll
  for (int e = 0; e < 9; e++) acc.e[e] = make_double2(0.0, 0.0);
  closers(acc, g, c, u, mu, cp, cr);
  M3 um, m, r;
  m_load(um, u + (size_t)mu * 9 * V, V, c.site);
  m_nn(m, um, acc);
  tah(r, m);
  m_store(f + (size_t)mu * 9 * V, V, c.site, r);
}

// sum_{x, mu>nu} Re Tr P and sum_{x, mu!=nu} Re Tr R (long side mu), each
// loop once, as Re Tr[U_mu(x) C] over the loops' first links
__global__ void __launch_bounds__(kBlock) gauge_action_kernel(Geom g, const double2 *__restrict__ u, int rect,
                                                              double *partials, unsigned *ticket, double *out) {
  double s[2] = {0.0, 0.0};
  const size_t V = (size_t)g.V;
  for (int site = blockIdx.x * blockDim.x + threadIdx.x; site < g.V; site += gridDim.x * blockDim.x) {
    SiteCtx c;
    c.site = site;
    c.par = site >= g.nh ? 1 : 0;
    site_coords(g, c.par, site - c.par * g.nh, c.x, c.lex);
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
      c.mu = mu;
#pragma unroll 1
      for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        PathCtx p{&g, &c, u, mu, nu};
        M3 t, um, m;
        m_load(um, u + (size_t)mu * 9 * V, V, site);
        if (nu < mu) {
          step_nu(t, p, 1, 0, 1, true);
          step_back_mu(t, p, 1, 1);
          step_nu(t, p, 0, 1, -1, false);
          m_nn(m, um, t);
          s[0] += m.e[0].x + m.e[4].x + m.e[8].x;
        }
        if (rect) {
          set_link(t, u + (size_t)mu * 9 * V, V, at(p, 1, 0), false);
          step_nu(t, p, 2, 0, 1, false);
          step_back_mu(t, p, 2, 1);
          step_back_mu(t, p, 1, 1);
          step_nu(t, p, 0, 1, -1, false);
          m_nn(m, um, t);
          s[1] += m.e[0].x + m.e[4].x + m.e[8].x;
        }
      }
    }
  }
  double tot[2];
  if (grid_reduce<2>(s, partials, ticket, tot) && threadIdx.x == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

// expAH(x): scale until |x|^2 <= 1/16, degree-12 Taylor polynomial in
// Paterson-Stockmeyer form (x, x^2, x^3), square back (matexp.nim:316-346)
__device__ __forceinline__ void exp_ah(M3 &r, const M3 &x0) {
  double n2 = 0.0;
#pragma unroll
  for (int e = 0; e < 9; e++) n2 += x0.e[e].x * x0.e[e].x + x0.e[e].y * x0.e[e].y;
  double scale = 1.0;
  int ns = 0;
  while (n2 > 1.0 / 16.0 && ns < 64) {
    n2 *= 0.25;
    scale *= 0.5;
    ns++;
  }
  M3 m = x0, m2, m3, a;
  m_scale(m, scale);
  m_nn(m2, m, m);
  m_nn(m3, m2, m);
  const double c2 = 0.5, c3 = 1.0 / 6, c4 = 1.0 / 24, c5 = 1.0 / 120, c6 = 1.0 / 720, c7 = 1.0 / 5040,
               c8 = 1.0 / 40320, c9 = 1.0 / 362880, c10 = 1.0 / 3628800, c11 = 1.0 / 39916800,
               c12 = 1.0 / 479001600;
  // a = c12 m3 + c11 m2 + c10 m + c9
#pragma unroll
  for (int e = 0; e < 9; e++)
    a.e[e] = make_double2(c12 * m3.e[e].x + c11 * m2.e[e].x + c10 * m.e[e].x,
                          c12 * m3.e[e].y + c11 * m2.e[e].y + c10 * m.e[e].y);
  a.e[0].x += c9;
  a.e[4].x += c9;
  a.e[8].x += c9;
  // a <- a m3 + c8 m2 + c7 m + c6, then + c5 m2 + c4 m + c3, then + c2 m2 + m + 1
  const double k2[3] = {c8, c5, c2}, k1[3] = {c7, c4, 1.0}, k0[3] = {c6, c3, 1.0};
#pragma unroll 1
  for (int s = 0; s < 3; s++) {
    m_nn(r, a, m3);
#pragma unroll
    for (int e = 0; e < 9; e++) {
      r.e[e].x += k2[s] * m2.e[e].x + k1[s] * m.e[e].x;
      r.e[e].y += k2[s] * m2.e[e].y + k1[s] * m.e[e].y;
    }
    r.e[0].x += k0[s];
    r.e[4].x += k0[s];
    r.e[8].x += k0[s];
    a = r;
  }
#pragma unroll 1
  for (int k = 0; k < ns; k++) {
    m_nn(r, a, a);
    a = r;
  }
  r = a;
}

__global__ void __launch_bounds__(kSmBlock) link_update_kernel(int V, double2 *u, const double2 *__restrict__ p,
                                                               double eps) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const size_t off = (size_t)blockIdx.y * 9 * V;
  M3 x, e, y, z;
  m_load(x, p + off, (size_t)V, s);
  m_scale(x, eps);
  exp_ah(e, x);
  m_load(y, u + off, (size_t)V, s);
  m_nn(z, e, y);
  m_store(u + off, (size_t)V, s, z);
}

__global__ void axpy_field_kernel(size_t n, double2 *y, double a, const double2 *__restrict__ x) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = x[i];
    double2 w = y[i];
    w.x = fma(a, v.x, w.x);
    w.y = fma(a, v.y, w.y);
    y[i] = w;
  }
}

// ---- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----
__device__ __forceinline__ uint4 philox4x32(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}
// uniform in (0, 1) from 64 random bits (53 used)
__device__ __forceinline__ double unit_open(uint32_t a, uint32_t b) {
  const uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);  // 53 bits
  return ((double)(v & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

// P = randTah3 per link (gaugeUtils.nim:1466-1493): Gaussian coefficients
// with the sqrt(1/2), sqrt(1/3) normalisation; link k of the field draws
// from counter (k, counter), key seed
__global__ void momenta_heatbath_kernel(int V, double2 *p, uint2 key, uint32_t clo, uint32_t chi) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V) return;
  const int mu = blockIdx.y;
  const uint32_t link = (uint32_t)mu * (uint32_t)V + (uint32_t)s;
  double gs[8];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const uint4 r0 = philox4x32(make_uint4(link, clo, chi, 2u * q), key);
    const uint4 r1 = philox4x32(make_uint4(link, clo, chi, 2u * q + 1u), key);
    const double u1 = unit_open(r0.x, r0.y), u2 = unit_open(r0.z, r0.w);
    const double u3 = unit_open(r1.x, r1.y), u4 = unit_open(r1.z, r1.w);
    const double ra = sqrt(-2.0 * log(u1)), rb = sqrt(-2.0 * log(u3));
    double sa, ca, sb, cb;
    sincospi(2.0 * u2, &sa, &ca);
    sincospi(2.0 * u4, &sb, &cb);
    gs[4 * q + 0] = ra * ca;
    gs[4 * q + 1] = ra * sa;
    gs[4 * q + 2] = rb * cb;
    gs[4 * q + 3] = rb * sb;
  }
  const double s2 = 0.70710678118654752440, s3 = 0.57735026918962576450;
  const double r3 = s2 * gs[0], r8 = s2 * s3 * gs[1];
  const double r01 = s2 * gs[2], r02 = s2 * gs[3], r12 = s2 * gs[4];
  const double i01 = s2 * gs[5], i02 = s2 * gs[6], i12 = s2 * gs[7];
  M3 m;
  m.e[0] = make_double2(0.0, r8 + r3);
  m.e[4] = make_double2(0.0, r8 - r3);
  m.e[8] = make_double2(0.0, -2.0 * r8);
  m.e[1] = make_double2(r01, i01);
  m.e[3] = make_double2(-r01, i01);
  m.e[2] = make_double2(r02, i02);
  m.e[6] = make_double2(-r02, i02);
  m.e[5] = make_double2(r12, i12);
  m.e[7] = make_double2(-r12, i12);
  m_store(p + (size_t)mu * 9 * V, (size_t)V, s, m);
}

__global__ void __launch_bounds__(kBlock) norm2_field_kernel(size_t n, const double2 *__restrict__ x, double *partials,
                                                             unsigned *ticket, double *out) {
  double s[1] = {0.0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = x[i];
    s[0] += v.x * v.x + v.y * v.y;
  }
  double tot[1];
  if (grid_reduce<1>(s, partials, ticket, tot) && threadIdx.x == 0) out[0] = tot[0];
}

// a 4-direction link field given in either memory space, staged on the
// device for host callers
struct Field4 {
  const Geom *g = nullptr;
  double2 *dev = nullptr;
  void *own = nullptr;
  double *host = nullptr;
  ~Field4() {
    if (own) {
      cudaStreamSynchronize(stream());
      cudaFree(own);
    }
  }
};

static int field_in(const Geom &g, const double *p, int mem, bool upload, Field4 &f) {
  f.g = &g;
  if (mem == QEXSTAG_MEM_DEVICE) {
    f.dev = (double2 *)p;
    return QEXSTAG_OK;
  }
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  if (cudaMalloc(&f.own, 5 * per) != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, "device allocation failed");
  }
  f.dev = (double2 *)f.own;
  f.host = (double *)p;
  if (upload) {
    double2 *aos = f.dev + 4 * 9 * (size_t)g.V;
    for (int d = 0; d < 4; d++) {
      QS_CUDA(cudaMemcpyAsync(aos, p + (size_t)d * 18 * g.V, per, cudaMemcpyHostToDevice, stream()));
      int rc = aos_to_soa((const double *)aos, f.dev + (size_t)d * 9 * g.V, g.V, g.V, 9);
      if (rc) return rc;
    }
  }
  return QEXSTAG_OK;
}

static int field_out(Field4 &f) {
  if (!f.own) return QEXSTAG_OK;
  const Geom &g = *f.g;
  const size_t per = sizeof(double2) * 9 * (size_t)g.V;
  double2 *aos = f.dev + 4 * 9 * (size_t)g.V;
  for (int d = 0; d < 4; d++) {
    int rc = soa_to_aos(f.dev + (size_t)d * 9 * g.V, (double *)aos, g.V, g.V, 9);
    if (rc) return rc;
    QS_CUDA(cudaMemcpyAsync(f.host + (size_t)d * 18 * g.V, aos, per, cudaMemcpyDeviceToHost, stream()));
  }
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

static int check_common(const qexstag_layout *l, int mem) {
  if (!l) return fail(QEXSTAG_ERR_ARG, "null layout");
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE) return fail(QEXSTAG_ERR_ARG, "bad memory kind");
  return runtime_ready();
}

static int read_results(int n, double *out) {
  QS_CUDA(cudaMemcpyAsync(host_results(), red_results(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  for (int i = 0; i < n; i++) out[i] = host_results()[i];
  return QEXSTAG_OK;
}

}  // namespace qs

using namespace qs;

extern "C" {

void qexstag_gauge_coefs_rect(qexstag_gauge_coefs *c, double beta, double c1) {
  if (!c) return;
  c->plaq = (1.0 - 8.0 * c1) * beta;
  c->rect = c1 * beta;
}

int qexstag_gauge_action(qexstag_layout *l, const qexstag_gauge_coefs *c, const double *u, int mem, double *action) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!c || !u || !action) return fail(QEXSTAG_ERR_ARG, "gauge_action: null argument");
  const Geom &g = l->g;
  Field4 U;
  if ((rc = field_in(g, u, mem, true, U))) return rc;
  const int grid = std::min(grid_for(g.V, kBlock, 8), kMaxRedBlocks * 8 / 2);
  gauge_action_kernel<<<grid, kBlock, 0, stream()>>>(g, U.dev, c->rect != 0.0 ? 1 : 0, red_partials(),
                                                     red_tickets(), red_results());
  note_launch();
  QS_LAUNCH_CHECK();
  double s[2];
  if ((rc = read_results(2, s))) return rc;
  *action = -(c->plaq * s[0] + c->rect * s[1]) / 3.0;
  return QEXSTAG_OK;
}

int qexstag_gauge_force(qexstag_layout *l, const qexstag_gauge_coefs *c, const double *u, double *f, int mem) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!c || !u || !f) return fail(QEXSTAG_ERR_ARG, "gauge_force: null argument");
  const Geom &g = l->g;
  Field4 U, Fo;
  if ((rc = field_in(g, u, mem, true, U)) || (rc = field_in(g, f, mem, false, Fo))) return rc;
  gauge_force_kernel<<<sweep_grid(g), kSmBlock, 0, stream()>>>(g, U.dev, Fo.dev, c->plaq / 3.0, c->rect / 3.0);
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = field_out(Fo))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_link_update(qexstag_layout *l, double *u, const double *p, double eps, int mem) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!u || !p) return fail(QEXSTAG_ERR_ARG, "link_update: null argument");
  if (!std::isfinite(eps)) return fail(QEXSTAG_ERR_ARG, "link_update: eps not finite");
  const Geom &g = l->g;
  Field4 U, P;
  if ((rc = field_in(g, u, mem, true, U)) || (rc = field_in(g, p, mem, true, P))) return rc;
  link_update_kernel<<<field_grid(g), kSmBlock, 0, stream()>>>(g.V, U.dev, P.dev, eps);
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = field_out(U))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_momenta_update(qexstag_layout *l, double *p, const double *f, double a, int mem) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!p || !f) return fail(QEXSTAG_ERR_ARG, "momenta_update: null argument");
  const Geom &g = l->g;
  Field4 P, Fi;
  if ((rc = field_in(g, p, mem, true, P)) || (rc = field_in(g, f, mem, true, Fi))) return rc;
  const size_t n = (size_t)36 * g.V;
  axpy_field_kernel<<<grid_for((long)std::min<size_t>(n, 1u << 30)), kBlock, 0, stream()>>>(n, P.dev, a, Fi.dev);
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = field_out(P))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_momenta_heatbath(qexstag_layout *l, double *p, unsigned long long seed, unsigned long long counter,
                             int mem) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!p) return fail(QEXSTAG_ERR_ARG, "momenta_heatbath: null argument");
  const Geom &g = l->g;
  if ((long long)4 * g.V > 0xffffffffll) return fail(QEXSTAG_ERR_ARG, "momenta_heatbath: lattice too large");
  Field4 P;
  if ((rc = field_in(g, p, mem, false, P))) return rc;
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  momenta_heatbath_kernel<<<field_grid(g), kSmBlock, 0, stream()>>>(g.V, P.dev, key, (uint32_t)counter,
                                                                    (uint32_t)(counter >> 32));
  note_launch();
  QS_LAUNCH_CHECK();
  if ((rc = field_out(P))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_kinetic_action(qexstag_layout *l, const double *p, int mem, double *t) {
  int rc;
  if ((rc = check_common(l, mem))) return rc;
  if (!p || !t) return fail(QEXSTAG_ERR_ARG, "kinetic_action: null argument");
  const Geom &g = l->g;
  Field4 P;
  if ((rc = field_in(g, p, mem, true, P))) return rc;
  const size_t n = (size_t)36 * g.V;
  const int grid = std::min(grid_for((long)std::min<size_t>(n, 1u << 30), kBlock, 8), kMaxRedBlocks * 8);
  norm2_field_kernel<<<grid, kBlock, 0, stream()>>>(n, P.dev, red_partials(), red_tickets(), red_results());
  note_launch();
  QS_LAUNCH_CHECK();
  double s;
  if ((rc = read_results(1, &s))) return rc;
  *t = 0.5 * s - 16.0 * (double)g.V;
  return QEXSTAG_OK;
}

}  // extern "C"
