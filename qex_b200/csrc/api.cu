// api.cu -- the extern "C" entry points declared in include/qexstag.h:
// argument checking, staging of host fields (QEX V=1 array-of-structs) to the
// device layout and back, and dispatch to the kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "lib.cuh"

namespace qs {

int build_low_links(qexstag_links_s *g);
void free_low_links(LowLinks &low);
int cgm_ee(qexstag_links_s *g, double m, int nshift, const double *sigma, int nrhs,
           const double2 *const *b, double2 *const *y, const qexstag_solver_params *p,
           qexstag_solver_stats *st, double *r2_out);
int solve_multishift(qexstag_links_s *g, int nmass, double2 *const *xs, const double2 *b,
                     const double *ms, const qexstag_solver_params *p, qexstag_solver_stats *st);
int apply_D(qexstag_links_s *g, double2 *r, const double2 *x, double m, double sc);
int stagD_par(qexstag_links_s *g, int par, double2 *r, const double2 *x, double m, double sc,
              double a);
int rephase_links(qexstag_links_s *g, bool literal);

int Workspace::get(int slot, size_t bytes, void **out) {
  auto it = bufs.find(slot);
  if (it != bufs.end() && it->second.first >= bytes) {
    *out = it->second.second;
    return QEXSTAG_OK;
  }
  if (it != bufs.end()) {
    cudaStreamSynchronize(stream());
    cudaFree(it->second.second);
    bufs.erase(it);
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(QEXSTAG_ERR_ALLOC, std::string("device allocation of ") + std::to_string(bytes) +
                                       " bytes failed: " + cudaGetErrorString(e));
  }
  bufs[slot] = std::make_pair(bytes, p);
  *out = p;
  return QEXSTAG_OK;
}

int Workspace::get_pinned(size_t bytes, void **out) {
  if (pinned && pinned_bytes >= bytes) {
    *out = pinned;
    return QEXSTAG_OK;
  }
  if (pinned) {
    cudaStreamSynchronize(stream());
    cudaFreeHost(pinned);
    pinned = nullptr;
  }
  cudaError_t e = cudaHostAlloc(&pinned, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    pinned = nullptr;
    return fail(QEXSTAG_ERR_ALLOC, "pinned host allocation failed");
  }
  pinned_bytes = bytes;
  *out = pinned;
  return QEXSTAG_OK;
}

void Workspace::release() {
  cudaStreamSynchronize(stream());
  for (auto &kv : bufs) cudaFree(kv.second.second);
  bufs.clear();
  if (pinned) cudaFreeHost(pinned);
  pinned = nullptr;
  pinned_bytes = 0;
}

// ---- staging of full-lattice colour vectors ----

// input: returns a device SoA [3][V] view of the field
static int stage_in(qexstag_links_s *g, int slot, const double *ptr, int mem,
                    const double2 **dev) {
  const Geom &geo = g->l->g;
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (const double2 *)ptr;
    return QEXSTAG_OK;
  }
  void *soa, *aos;
  const size_t bytes = sizeof(double2) * 3 * (size_t)geo.V;
  int rc;
  if ((rc = g->ws.get(slot, bytes, &soa)) || (rc = g->ws.get(kSlotAos, bytes, &aos))) return rc;
  QS_CUDA(cudaMemcpyAsync(aos, ptr, bytes, cudaMemcpyHostToDevice, stream()));
  if ((rc = aos_to_soa((const double *)aos, (double2 *)soa, geo.V, geo.V, 3))) return rc;
  *dev = (const double2 *)soa;
  return QEXSTAG_OK;
}

// parity block par of a host field (QEX V=1 order: the nh sites of parity 0
// first) into block par of a SoA slot; the slot's other block is not
// written (the caller reads block par only)
static int stage_in_block(qexstag_links_s *g, int slot, const double *ptr, int mem, int par,
                          const double2 **dev) {
  const Geom &geo = g->l->g;
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (const double2 *)ptr;
    return QEXSTAG_OK;
  }
  void *soa, *aos;
  const size_t bytes = sizeof(double2) * 3 * (size_t)geo.V;
  const size_t half = sizeof(double2) * 3 * (size_t)geo.nh;
  int rc;
  if ((rc = g->ws.get(slot, bytes, &soa)) || (rc = g->ws.get(kSlotAos, bytes, &aos))) return rc;
  QS_CUDA(cudaMemcpyAsync((char *)aos + par * half, (const char *)ptr + par * half, half, cudaMemcpyHostToDevice,
                          stream()));
  if ((rc = aos_to_soa((const double *)aos + (size_t)par * 6 * geo.nh, (double2 *)soa + (size_t)par * geo.nh,
                       geo.nh, geo.V, 3)))
    return rc;
  *dev = (const double2 *)soa;
  return QEXSTAG_OK;
}

static int stage_out_buf(qexstag_links_s *g, int slot, double *ptr, int mem, double2 **dev) {
  const Geom &geo = g->l->g;
  if (mem == QEXSTAG_MEM_DEVICE) {
    *dev = (double2 *)ptr;
    return QEXSTAG_OK;
  }
  void *soa;
  int rc = g->ws.get(slot, sizeof(double2) * 3 * (size_t)geo.V, &soa);
  if (rc) return rc;
  *dev = (double2 *)soa;
  return QEXSTAG_OK;
}

static int stage_out_finish(qexstag_links_s *g, const double2 *dev, double *ptr, int mem) {
  if (mem == QEXSTAG_MEM_DEVICE) return QEXSTAG_OK;
  const Geom &geo = g->l->g;
  void *aos;
  const size_t bytes = sizeof(double2) * 3 * (size_t)geo.V;
  int rc = g->ws.get(kSlotAos, bytes, &aos);
  if (rc) return rc;
  if ((rc = soa_to_aos(dev, (double *)aos, geo.V, geo.V, 3))) return rc;
  QS_CUDA(cudaMemcpyAsync(ptr, aos, bytes, cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

static int check_links(const qexstag_links_s *g) {
  if (!g || !g->l || !g->u64) return fail(QEXSTAG_ERR_ARG, "null or destroyed link handle");
  int d = -1;
  cudaGetDevice(&d);
  if (d != g->l->device) return fail(QEXSTAG_ERR_STATE, "link handle belongs to another device");
  return runtime_ready();
}

static int check_mem(int mem) {
  if (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE)
    return fail(QEXSTAG_ERR_ARG, "mem must be QEXSTAG_MEM_HOST or QEXSTAG_MEM_DEVICE");
  return QEXSTAG_OK;
}

struct Timer {
  cudaEvent_t a, b;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, stream());
  }
  double seconds() {
    cudaEventRecord(b, stream());
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3;
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

static void init_stats(qexstag_solver_stats *st) {
  std::memset(st, 0, sizeof(*st));
  st->calls = 1;
  st->kernel_launches = -launch_count();  // completed by finish_stats
}
static void finish_stats(qexstag_solver_stats *st) { st->kernel_launches += launch_count(); }
static double geo_nh(const qexstag_links_s *g) { return (double)g->l->g.nh; }

}  // namespace qs

using namespace qs;

extern "C" {

// ---------------------------------------------------------------------------
// layout
// ---------------------------------------------------------------------------

int qexstag_layout_create(const int dims[4], qexstag_layout **out) {
  if (!dims || !out) return fail(QEXSTAG_ERR_ARG, "layout_create: null argument");
  long V = 1;
  for (int d = 0; d < 4; d++) {
    if (dims[d] < 4 || (dims[d] & 1))
      return fail(QEXSTAG_ERR_ARG, "layout_create: every dimension must be even and >= 4");
    V *= dims[d];
  }
  if (V * 9 * 8 >= (1L << 31) * 1L && V >= (1L << 28))
    return fail(QEXSTAG_ERR_ARG, "layout_create: lattice too large");
  int rc = runtime_ready();
  if (rc) return rc;
  qexstag_layout_s *l = new (std::nothrow) qexstag_layout_s;
  if (!l) return fail(QEXSTAG_ERR_ALLOC, "layout_create: out of host memory");
  for (int d = 0; d < 4; d++) l->g.L[d] = dims[d];
  l->g.stride[0] = 1;
  for (int d = 1; d < 4; d++) l->g.stride[d] = l->g.stride[d - 1] * dims[d - 1];
  l->g.V = (int)V;
  l->g.nh = (int)(V / 2);
  l->g.t0 = 0;
  l->g.L3g = dims[3];
  set_fastdiv(l->g);
  cudaGetDevice(&l->device);
  *out = l;
  return QEXSTAG_OK;
}

int qexstag_layout_destroy(qexstag_layout *l) {
  delete l;
  return QEXSTAG_OK;
}

int qexstag_layout_index(const qexstag_layout *l, const int x[4], int64_t *idx) {
  if (!l || !x || !idx) return fail(QEXSTAG_ERR_ARG, "layout_index: null argument");
  const Geom &g = l->g;
  long lex = 0, p = 0;
  for (int d = 3; d >= 0; d--) {
    if (x[d] < 0 || x[d] >= g.L[d]) return fail(QEXSTAG_ERR_ARG, "layout_index: coordinate out of range");
    lex = lex * g.L[d] + x[d];
    p += x[d];
  }
  *idx = (lex + ((p & 1) ? g.V : 0)) / 2;
  return QEXSTAG_OK;
}

}  // extern "C"

namespace qs {
__global__ void shift_table_kernel(Geom g, int mu, int len, int par, int n, int32_t *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = par == 2 ? (i >= g.nh ? 1 : 0) : par;
    int k = par == 2 ? i - p * g.nh : i;
    int x[4], lex;
    site_coords(g, p, k, x, lex);
    out[i] = (1 - p) * g.nh + nbr_half(g, x, lex, mu, len);
  }
}
}  // namespace qs

extern "C" {

int qexstag_layout_shift_table(const qexstag_layout *l, int mu, int len, int subset,
                               int32_t *out_host) {
  if (!l || !out_host) return fail(QEXSTAG_ERR_ARG, "shift_table: null argument");
  if (mu < 0 || mu > 3 || subset < 0 || subset > 2)
    return fail(QEXSTAG_ERR_ARG, "shift_table: bad direction or subset");
  if ((len & 1) == 0 || len > 3 || len < -3)
    return fail(QEXSTAG_ERR_ARG, "shift_table: len must be +-1 or +-3");
  int rc = runtime_ready();
  if (rc) return rc;
  const Geom &g = l->g;
  int n = subset == 2 ? g.V : g.nh;
  int32_t *d = nullptr;
  QS_CUDA(cudaMalloc(&d, sizeof(int32_t) * n));
  shift_table_kernel<<<grid_for(n), kBlock, 0, stream()>>>(g, mu, len, subset, n, d);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, d, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, stream());
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "shift_table");
  return QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// links
// ---------------------------------------------------------------------------

}  // extern "C"

namespace qs {
// copy a link list into g->u64 (host AoS layout or device SoA layout)
static int upload_links(qexstag_links_s *g, const double *links, int mem) {
  const Geom &geo = g->l->g;
  const size_t per = sizeof(double2) * 9 * (size_t)geo.V;
  if (mem == QEXSTAG_MEM_DEVICE) {
    QS_CUDA(cudaMemcpyAsync(g->u64, links, per * g->nl, cudaMemcpyDeviceToDevice, stream()));
    return QEXSTAG_OK;
  }
  void *aos;
  int rc = g->ws.get(kSlotAos, per, &aos);
  if (rc) return rc;
  for (int k = 0; k < g->nl; k++) {
    QS_CUDA(cudaMemcpyAsync(aos, links + (size_t)k * 18 * geo.V, per, cudaMemcpyHostToDevice, stream()));
    if ((rc = aos_to_soa((const double *)aos, g->u64 + (size_t)k * 9 * geo.V, geo.V, geo.V, 9))) return rc;
  }
  return QEXSTAG_OK;
}
// MILC order (QUDA_MILC_GAUGE_ORDER): a site's four directions together,
// double[V][4][3][3][2] per list.  kind 0: the naive list (slot mu), 1: fat
// links of a fat+Naik list (slot 2 mu), 2: its long links (slot 2 mu + 1).
// Sites [s0, s0 + n) pass through aos, n * 4 * 9 double2.
__global__ void milc_soa_kernel(double2 *__restrict__ aos, double2 *__restrict__ soa, int V, int s0, int n, int kind,
                                int to_soa) {
  const int ss = kind == 0 ? 1 : 2, so = kind == 2 ? 1 : 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * 36; t += gridDim.x * blockDim.x) {
    const int i = t / 36, r = t - i * 36, mu = r / 9, c = r - mu * 9;
    double2 *d = soa + ((size_t)(mu * ss + so) * 9 + c) * V + s0 + i;
    if (to_soa)
      *d = aos[t];
    else
      aos[t] = *d;
  }
}

static int milc_transfer(qexstag_links_s *g, double *host, int kind, bool up) {
  const Geom &geo = g->l->g;
  const size_t per = sizeof(double2) * 9 * (size_t)geo.V;  // staging: V/4 sites of 4 directions
  void *aos;
  int rc = g->ws.get(kSlotAos, per, &aos);
  if (rc) return rc;
  const int chunk = geo.V / 4;
  for (int s0 = 0; s0 < geo.V; s0 += chunk) {
    const int n = std::min(chunk, geo.V - s0);
    double *h = host + (size_t)s0 * 4 * 18;
    const size_t bytes = sizeof(double2) * 36 * (size_t)n;
    if (up) QS_CUDA(cudaMemcpyAsync(aos, h, bytes, cudaMemcpyHostToDevice, stream()));
    milc_soa_kernel<<<grid_for((long)n * 36), kBlock, 0, stream()>>>((double2 *)aos, g->u64, geo.V, s0, n, kind,
                                                                        up ? 1 : 0);
    note_launch();
    QS_LAUNCH_CHECK();
    if (!up) {
      QS_CUDA(cudaMemcpyAsync(h, aos, bytes, cudaMemcpyDeviceToHost, stream()));
      QS_CUDA(cudaStreamSynchronize(stream()));  // the staging buffer is reused by the next chunk
    }
  }
  return QEXSTAG_OK;
}

static int upload_links_milc(qexstag_links_s *g, const double *fat, const double *lng) {
  int rc = milc_transfer(g, const_cast<double *>(fat), g->nl == 8 ? 1 : 0, true);
  if (!rc && g->nl == 8) rc = milc_transfer(g, const_cast<double *>(lng), 2, true);
  return rc;
}

static int download_links_milc(qexstag_links_s *g, double *fat, double *lng) {
  int rc = milc_transfer(g, fat, g->nl == 8 ? 1 : 0, false);
  if (!rc && g->nl == 8) rc = milc_transfer(g, lng, 2, false);
  return rc;
}
}  // namespace qs

extern "C" {

int qexstag_links_create(qexstag_layout *l, int nlinks, const double *links, int mem,
                         double long_coeff, qexstag_links **out) {
  if (!l || !links || !out) return fail(QEXSTAG_ERR_ARG, "links_create: null argument");
  if (nlinks != 4 && nlinks != 8) return fail(QEXSTAG_ERR_ARG, "links_create: nlinks must be 4 or 8");
  int rc;
  if ((rc = check_mem(mem)) || (rc = runtime_ready())) return rc;
  if (long_coeff == 0.0 || !std::isfinite(long_coeff))
    return fail(QEXSTAG_ERR_ARG, "links_create: long_coeff must be finite and nonzero");
  qexstag_links_s *g = new (std::nothrow) qexstag_links_s;
  if (!g) return fail(QEXSTAG_ERR_ALLOC, "links_create: out of host memory");
  g->l = l;
  g->nl = nlinks;
  g->long_coeff = long_coeff;
  const Geom &geo = l->g;
  const size_t per = sizeof(double2) * 9 * (size_t)geo.V;
  cudaError_t e = cudaMalloc(&g->u64, per * nlinks);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete g;
    return fail(QEXSTAG_ERR_ALLOC, "links_create: device allocation failed");
  }
  if ((rc = upload_links(g, links, mem))) {
    g->ws.release();
    cudaFree(g->u64);
    delete g;
    return rc;
  }
  if ((rc = build_low_links(g))) {
    g->ws.release();
    free_low_links(g->low);
    cudaFree(g->u64);
    delete g;
    return rc;
  }
  e = cudaStreamSynchronize(stream());
  if (e != cudaSuccess) return cuda_fail(e, "links_create");
  *out = g;
  return QEXSTAG_OK;
}

int qexstag_links_update(qexstag_links *g, const double *links, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!links) return fail(QEXSTAG_ERR_ARG, "links_update: null links");
  if ((rc = upload_links(g, links, mem))) return rc;
  free_low_links(g->low);
  if ((rc = build_low_links(g))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_rephase(qexstag_links *g) {
  int rc;
  if ((rc = check_links(g))) return rc;
  if ((rc = rephase_links(g, true))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_rephase_all(qexstag_links *g) {
  int rc;
  if ((rc = check_links(g))) return rc;
  if ((rc = rephase_links(g, false))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_create_milc(qexstag_layout *l, const double *fat, const double *lng, double long_coeff,
                              qexstag_links **out) {
  if (!l || !fat || !out) return fail(QEXSTAG_ERR_ARG, "links_create_milc: null argument");
  int rc;
  if ((rc = runtime_ready())) return rc;
  if (long_coeff == 0.0 || !std::isfinite(long_coeff))
    return fail(QEXSTAG_ERR_ARG, "links_create_milc: long_coeff must be finite and nonzero");
  const int nl = lng ? 8 : 4;
  qexstag_links_s *g = new (std::nothrow) qexstag_links_s;
  if (!g) return fail(QEXSTAG_ERR_ALLOC, "links_create_milc: out of host memory");
  g->l = l;
  g->nl = nl;
  g->long_coeff = long_coeff;
  const size_t per = sizeof(double2) * 9 * (size_t)l->g.V;
  cudaError_t e = cudaMalloc(&g->u64, per * nl);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete g;
    return fail(QEXSTAG_ERR_ALLOC, "links_create_milc: device allocation failed");
  }
  if ((rc = upload_links_milc(g, fat, lng)) || (rc = build_low_links(g))) {
    g->ws.release();
    free_low_links(g->low);
    cudaFree(g->u64);
    delete g;
    return rc;
  }
  e = cudaStreamSynchronize(stream());
  if (e != cudaSuccess) return cuda_fail(e, "links_create_milc");
  *out = g;
  return QEXSTAG_OK;
}

int qexstag_links_update_milc(qexstag_links *g, const double *fat, const double *lng) {
  int rc;
  if ((rc = check_links(g))) return rc;
  if (!fat || ((g->nl == 8) != (lng != nullptr)))
    return fail(QEXSTAG_ERR_ARG, "links_update_milc: fat is null, or lng is given for a naive handle "
                                 "or missing for a fat+Naik handle");
  if ((rc = upload_links_milc(g, fat, lng))) return rc;
  free_low_links(g->low);
  if ((rc = build_low_links(g))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_get_milc(qexstag_links *g, double *fat, double *lng) {
  int rc;
  if ((rc = check_links(g))) return rc;
  if (!fat || ((g->nl == 8) != (lng != nullptr)))
    return fail(QEXSTAG_ERR_ARG, "links_get_milc: fat is null, or lng is given for a naive handle "
                                 "or missing for a fat+Naik handle");
  if ((rc = download_links_milc(g, fat, lng))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_links_destroy(qexstag_links *g) {
  if (!g) return QEXSTAG_OK;
  g->ws.release();
  free_low_links(g->low);
  cudaFree(g->u64);
  g->u64 = nullptr;
  delete g;
  return QEXSTAG_OK;
}

int qexstag_links_recon12(const qexstag_links *g) { return (g && g->low.recon12) ? 1 : 0; }

// ---------------------------------------------------------------------------
// Dslash entry points
// ---------------------------------------------------------------------------

int qexstag_stagD2(qexstag_links *g, int subset, double *r, const double *x, double a, double b,
                   int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "stagD2: null field");
  if (subset != QEXSTAG_EVEN && subset != QEXSTAG_ODD)
    return fail(QEXSTAG_ERR_ARG, "stagD2: subset must be EVEN or ODD");
  const Geom &geo = g->l->g;
  const double2 *dx, *dr_in = nullptr;
  double2 *dr;
  if ((rc = stage_in(g, kSlotIn0, x, mem, &dx))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, r, mem, &dr))) return rc;
  if (mem == QEXSTAG_MEM_HOST) {
    // r is an input where it is not overwritten: stage all of it
    if ((rc = stage_in(g, kSlotOut0, r, mem, &dr_in))) return rc;
  }
  const int init = (a == 0.0 && b == 0.0) ? 0 : (a == 0.0 ? 1 : 2);
  rc = dslash64(g, subset, block(dr, geo, subset), block(dx, geo, 1 - subset), block(dx, geo, subset),
                block((const double2 *)dr, geo, subset), a, b, 1.0, +1, init);
  if (rc) return rc;
  return stage_out_finish(g, dr, r, mem);
}

int qexstag_stagDN(qexstag_links *g, int subset, int n, double *const *r, const double *const *x, double m,
                   int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (n < 1 || !r || !x) return fail(QEXSTAG_ERR_ARG, "stagDN: n must be >= 1 with r and x given");
  for (int i = 0; i < n; i++)
    if (!r[i] || !x[i]) return fail(QEXSTAG_ERR_ARG, "stagDN: null field");
  if (subset != QEXSTAG_EVEN && subset != QEXSTAG_ODD)
    return fail(QEXSTAG_ERR_ARG, "stagDN: subset must be EVEN or ODD");
  const Geom &geo = g->l->g;
  if (mem == QEXSTAG_MEM_DEVICE)
    return dslashN64(g, subset, n, (double2 *const *)r, geo.V, (const double2 *const *)x, geo.V, m);
  // host fields: 8 at a time through the staging slots; r is staged in whole
  // so that its other parity comes back unchanged
  for (int i0 = 0; i0 < n; i0 += 8) {
    const int nb = std::min(8, n - i0);
    const double2 *dx[8];
    double2 *dr[8];
    for (int j = 0; j < nb; j++) {
      const double2 *t;
      if ((rc = stage_in(g, kSlotDn0 + j, x[i0 + j], mem, &dx[j])) ||
          (rc = stage_in(g, kSlotDn0 + 8 + j, r[i0 + j], mem, &t)))
        return rc;
      dr[j] = const_cast<double2 *>(t);
    }
    if ((rc = dslashN64(g, subset, nb, dr, geo.V, dx, geo.V, m))) return rc;
    for (int j = 0; j < nb; j++)
      if ((rc = stage_out_finish(g, dr[j], r[i0 + j], mem))) return rc;
  }
  return QEXSTAG_OK;
}

static int stagD_api(qexstag_links *g, int subset, double *r, const double *x, double m, double sc,
                     double a, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "stagD: null field");
  if (subset < 0 || subset > 2) return fail(QEXSTAG_ERR_ARG, "stagD: bad subset");
  if (sc == 0.0) return fail(QEXSTAG_ERR_ARG, "stagD: sc must be nonzero");
  const double2 *dx, *dr_in;
  double2 *dr;
  if ((rc = stage_in(g, kSlotIn0, x, mem, &dx))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, r, mem, &dr))) return rc;
  if (mem == QEXSTAG_MEM_HOST && (subset != 2 || a != 0.0)) {
    if ((rc = stage_in(g, kSlotOut0, r, mem, &dr_in))) return rc;
  }
  if (subset == 2) {
    if ((rc = stagD_par(g, 0, dr, dx, m, sc, a))) return rc;
    if ((rc = stagD_par(g, 1, dr, dx, m, sc, a))) return rc;
  } else {
    if ((rc = stagD_par(g, subset, dr, dx, m, sc, a))) return rc;
  }
  return stage_out_finish(g, dr, r, mem);
}

int qexstag_stagD(qexstag_links *g, int subset, double *r, const double *x, double m, double sc,
                  double a, int mem) {
  return stagD_api(g, subset, r, x, m, sc, a, mem);
}
int qexstag_D(qexstag_links *g, double *r, const double *x, double m, int mem) {
  return stagD_api(g, 2, r, x, m, 1.0, 0.0, mem);
}
int qexstag_Ddag(qexstag_links *g, double *r, const double *x, double m, int mem) {
  return stagD_api(g, 2, r, x, m, -1.0, 0.0, mem);
}

static int schur_api(qexstag_links *g, int par, double *r, const double *x, double m2, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "stagD2ee: null field");
  const Geom &geo = g->l->g;
  const double2 *dx, *dr_in;
  double2 *dr;
  void *pt;
  if ((rc = stage_in(g, kSlotIn0, x, mem, &dx))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, r, mem, &dr))) return rc;
  if (mem == QEXSTAG_MEM_HOST) {
    if ((rc = stage_in(g, kSlotOut0, r, mem, &dr_in))) return rc;
  }
  if ((rc = g->ws.get(kSlotTmpOdd, sizeof(double2) * 3 * (size_t)geo.nh, &pt))) return rc;
  if ((rc = schur64(g, par, block(dr, geo, par), block(dx, geo, par), VecD{(double2 *)pt, geo.nh}, m2)))
    return rc;
  return stage_out_finish(g, dr, r, mem);
}

int qexstag_stagD2ee(qexstag_links *g, double *r, const double *x, double m2, int mem) {
  return schur_api(g, 0, r, x, m2, mem);
}
int qexstag_stagD2oo(qexstag_links *g, double *r, const double *x, double m2, int mem) {
  return schur_api(g, 1, r, x, m2, mem);
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------

static int check_params(const qexstag_solver_params *p) {
  if (!p) return fail(QEXSTAG_ERR_ARG, "null solver params");
  if (!(p->r2req >= 0.0) || !std::isfinite(p->r2req)) return fail(QEXSTAG_ERR_ARG, "r2req must be >= 0");
  if (p->sloppy < 0 || p->sloppy > 2) return fail(QEXSTAG_ERR_ARG, "sloppy must be 0, 1 or 2");
  return QEXSTAG_OK;
}

static int solveXX_api(qexstag_links *g, int par, double *r, const double *x, double m,
                       const qexstag_solver_params *p, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "solveXX: null field");
  qexstag_solver_stats st;
  init_stats(&st);
  const double2 *dx;
  double2 *dr;
  Timer tm;
  // solveXX reads x on parity par only
  if ((rc = stage_in_block(g, kSlotIn0, x, mem, par, &dx))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, r, mem, &dr))) return rc;
  int status = solve_xx(g, par, dr, dx, m, p, &st);
  if (status < 0) return status;
  if ((rc = stage_out_finish(g, dr, r, mem))) return rc;
  st.seconds = tm.seconds();
  st.flops = (double)(g->nl * 4 * 72 + 60) * g->l->g.nh * st.iterations;
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

int qexstag_solveEE(qexstag_links *g, double *r, const double *x, double m,
                    const qexstag_solver_params *p, qexstag_solver_stats *st, int mem) {
  return solveXX_api(g, 0, r, x, m, p, st, mem);
}
int qexstag_solveOO(qexstag_links *g, double *r, const double *x, double m,
                    const qexstag_solver_params *p, qexstag_solver_stats *st, int mem) {
  return solveXX_api(g, 1, r, x, m, p, st, mem);
}

int qexstag_solve(qexstag_links *g, double *x, const double *b, double m,
                  const qexstag_solver_params *p, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (!x || !b) return fail(QEXSTAG_ERR_ARG, "solve: null field");
  qexstag_solver_stats st;
  init_stats(&st);
  const double2 *db;
  double2 *dx;
  Timer tm;
  if ((rc = stage_in(g, kSlotIn0, b, mem, &db))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, x, mem, &dx))) return rc;
  if (mem == QEXSTAG_MEM_HOST && p->use_prev_soln) {
    const double2 *tmp;
    if ((rc = stage_in(g, kSlotOut0, x, mem, &tmp))) return rc;
  }
  int status = solve_full(g, dx, db, m, p, &st);
  if (status < 0) return status;
  if ((rc = stage_out_finish(g, dx, x, mem))) return rc;
  st.seconds = tm.seconds();
  st.flops = (double)(g->nl * 4 * 72 + 60) * g->l->g.nh * st.iterations +
             (double)(g->nl * 4 * 72 + 24) * g->l->g.nh;
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

int qexstag_solve_multishift(qexstag_links *g, int nmass, double *const *xs, const double *b,
                             const double *ms, const qexstag_solver_params *p,
                             qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (nmass < 1 || nmass > 64 || !xs || !b || !ms)
    return fail(QEXSTAG_ERR_ARG, "solve_multishift: need 1..64 masses and non-null fields");
  for (int k = 0; k < nmass; k++)
    if (!xs[k]) return fail(QEXSTAG_ERR_ARG, "solve_multishift: null output field");
  const Geom &geo = g->l->g;
  qexstag_solver_stats st;
  init_stats(&st);
  Timer tm;
  const double2 *db;
  if ((rc = stage_in(g, kSlotIn0, b, mem, &db))) return rc;
  double2 *dxs[64];
  for (int k = 0; k < nmass; k++) {
    if (mem == QEXSTAG_MEM_DEVICE) {
      dxs[k] = (double2 *)xs[k];
    } else {
      void *q;
      if ((rc = g->ws.get(kSlotMs0 + 100 + k, sizeof(double2) * 3 * (size_t)geo.V, &q))) return rc;
      dxs[k] = (double2 *)q;
    }
  }
  int status = solve_multishift(g, nmass, dxs, db, ms, p, &st);
  if (status < 0) return status;
  for (int k = 0; k < nmass; k++)
    if ((rc = stage_out_finish(g, dxs[k], xs[k], mem))) return rc;
  st.seconds = tm.seconds();
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

int qexstag_cgm_ee(qexstag_links *g, double m, int nshift, const double *sigma, int nrhs,
                   const double *const *b, double *const *y, const qexstag_solver_params *p,
                   qexstag_solver_stats *st_out, double *r2_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (nshift < 1 || nshift > 32 || nrhs < 1 || nrhs > 16 || !sigma || !b || !y)
    return fail(QEXSTAG_ERR_ARG, "cgm_ee: need 1..32 shifts, 1..16 right-hand sides");
  for (int k = 0; k < nshift; k++)
    if (!(sigma[k] >= 0.0)) return fail(QEXSTAG_ERR_ARG, "cgm_ee: shifts must be >= 0");
  const Geom &geo = g->l->g;
  qexstag_solver_stats st;
  init_stats(&st);
  Timer tm;
  const size_t fb = sizeof(double2) * 3 * (size_t)geo.V;
  const double2 *db[16];
  double2 *dy[16 * 32];
  for (int j = 0; j < nrhs; j++) {
    if (!b[j]) return fail(QEXSTAG_ERR_ARG, "cgm_ee: null right-hand side");
    if ((rc = stage_in(g, kSlotMs0 + j, b[j], mem, &db[j]))) return rc;
  }
  for (int i = 0; i < nrhs * nshift; i++) {
    if (!y[i]) return fail(QEXSTAG_ERR_ARG, "cgm_ee: null solution field");
    if (mem == QEXSTAG_MEM_DEVICE) {
      dy[i] = (double2 *)y[i];
    } else {
      void *q;
      if ((rc = g->ws.get(kSlotLast + i, fb, &q))) return rc;
      dy[i] = (double2 *)q;
    }
  }
  int status = cgm_ee(g, m, nshift, sigma, nrhs, db, dy, p, &st, r2_out);
  if (status < 0) return status;
  for (int i = 0; i < nrhs * nshift; i++)
    if ((rc = stage_out_finish(g, dy[i], y[i], mem))) return rc;
  st.seconds = tm.seconds();
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

}  // extern "C"

namespace qs {
int solve_batched(int nprob, qexstag_links_s *const *gs, const double *mass, double2 *const *x,
                  const double2 *const *b, const qexstag_solver_params *p, int *iters, double *r2_out,
                  qexstag_solver_stats *st, int *tuned_block, int *tuned_per_sm, int *graph_used);
}

extern "C" {

int qexstag_solve_batched(int nprob, qexstag_links *const *g, const double *mass, double *const *x,
                          const double *const *b, const qexstag_solver_params *p, int *iterations,
                          double *r2_out, int *launch_info, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (nprob < 1 || nprob > 128 || !g || !mass || !x || !b || !iterations)
    return fail(QEXSTAG_ERR_ARG, "solve_batched: need 1..128 problems and non-null arrays");
  if (p->sloppy != QEXSTAG_SLOPPY_NONE)
    return fail(QEXSTAG_ERR_ARG, "solve_batched: the batched persistent solver is FP64 (sloppy NONE)");
  for (int j = 0; j < nprob; j++) {
    if ((rc = check_links(g[j]))) return rc;
    if (g[j]->nl != g[0]->nl) return fail(QEXSTAG_ERR_ARG, "solve_batched: all problems need the same nlinks");
    if (!x[j] || !b[j]) return fail(QEXSTAG_ERR_ARG, "solve_batched: null field");
    for (int i = 0; i < j; i++)
      if (g[i] == g[j]) return fail(QEXSTAG_ERR_ARG, "solve_batched: one link handle per problem");
  }
  qexstag_solver_stats st;
  init_stats(&st);
  Timer tm;
  std::vector<const double2 *> db(nprob);
  std::vector<double2 *> dx(nprob);
  for (int j = 0; j < nprob; j++) {
    if ((rc = stage_in(g[j], kSlotIn0, b[j], mem, &db[j]))) return rc;
    if ((rc = stage_out_buf(g[j], kSlotOut0, x[j], mem, &dx[j]))) return rc;
    const Geom &geo = g[j]->l->g;
    if ((rc = vzero(VecD{dx[j] + geo.nh, geo.V}, geo.nh))) return rc;  // odd sites: 0 (solveEE)
  }
  std::vector<double2 *> xe(nprob);
  std::vector<const double2 *> be(nprob);
  for (int j = 0; j < nprob; j++) {
    xe[j] = dx[j];
    be[j] = db[j];
  }
  int blk = 0, per_sm = 0, graph = 0;
  int status = solve_batched(nprob, g, mass, xe.data(), be.data(), p, iterations, r2_out, &st, &blk, &per_sm,
                             &graph);
  if (status < 0) return status;
  for (int j = 0; j < nprob; j++)
    if ((rc = stage_out_finish(g[j], dx[j], x[j], mem))) return rc;
  st.seconds = tm.seconds();
  double fl = 0;
  for (int j = 0; j < nprob; j++) fl += (double)(g[j]->nl * 4 * 72 + 60) * g[j]->l->g.nh * iterations[j];
  st.flops = fl;
  finish_stats(&st);
  if (launch_info) {
    launch_info[0] = blk;
    launch_info[1] = per_sm;
    launch_info[2] = graph;
  }
  if (st_out) *st_out = st;
  return status;
}

// ---------------------------------------------------------------------------
// force
// ---------------------------------------------------------------------------

static int force_out(qexstag_links *g, double2 *df, double *f, int mem) {
  if (mem == QEXSTAG_MEM_DEVICE) return QEXSTAG_OK;
  const Geom &geo = g->l->g;
  const size_t per = sizeof(double2) * 9 * (size_t)geo.V;
  void *aos;
  int rc = g->ws.get(kSlotAos, per, &aos);
  if (rc) return rc;
  for (int k = 0; k < g->nl; k++) {
    if ((rc = soa_to_aos(df + (size_t)k * 9 * geo.V, (double *)aos, geo.V, geo.V, 9))) return rc;
    QS_CUDA(cudaMemcpyAsync(f + (size_t)k * 18 * geo.V, aos, per, cudaMemcpyDeviceToHost, stream()));
  }
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

static int force_buf(qexstag_links *g, double *f, int mem, double2 **df) {
  if (mem == QEXSTAG_MEM_DEVICE) {
    *df = (double2 *)f;
    return QEXSTAG_OK;
  }
  void *q;
  int rc = g->ws.get(kSlotLast + 600, sizeof(double2) * 9 * (size_t)g->l->g.V * g->nl, &q);
  *df = (double2 *)q;
  return rc;
}

int qexstag_ferm_force(qexstag_links *g, double *f, const double *psi, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!f || !psi) return fail(QEXSTAG_ERR_ARG, "ferm_force: null field");
  const double2 *dpsi;
  double2 *df;
  if ((rc = stage_in(g, kSlotIn0, psi, mem, &dpsi))) return rc;
  if ((rc = force_buf(g, f, mem, &df))) return rc;
  if ((rc = ferm_force64(g, df, dpsi))) return rc;
  return force_out(g, df, f, mem);
}

int qexstag_ferm_outer(qexstag_links *g, double *f, const double *psi, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem))) return rc;
  if (!f || !psi) return fail(QEXSTAG_ERR_ARG, "ferm_outer: null field");
  const double2 *dpsi;
  double2 *df;
  if ((rc = stage_in(g, kSlotIn0, psi, mem, &dpsi))) return rc;
  if ((rc = force_buf(g, f, mem, &df))) return rc;
  if ((rc = ferm_outer64(g, df, dpsi))) return rc;
  return force_out(g, df, f, mem);
}

// stagForceSolve (hmcAction.nim:669-721) into a full-lattice psi
static int force_solve_dev(qexstag_links *g, double2 *psi, const double2 *phi, double m,
                           const qexstag_solver_params *p, qexstag_solver_stats *st) {
  const Geom &geo = g->l->g;
  void *pvar;
  int rc;
  if ((rc = g->ws.get(kSlotFull1, sizeof(double2) * 3 * (size_t)geo.V, &pvar))) return rc;
  double2 *varphi = (double2 *)pvar;
  int status = solve_xx(g, 0, varphi, phi, m, p, st);
  if (status < 0) return status;
  if ((rc = vscale(block(varphi, geo, 0), 4.0, geo.nh))) return rc;
  // psi_o = (2D)_oe varphi_e (stagD2 with a = b = 0); psi_e = varphi_e
  if ((rc = dslash64(g, 1, block(psi, geo, 1), block((const double2 *)varphi, geo, 0), CVecD{nullptr, 0},
                     CVecD{nullptr, 0}, 0.0, 0.0, 1.0, +1, 0)))
    return rc;
  if ((rc = vcopy(block(psi, geo, 0), block((const double2 *)varphi, geo, 0), geo.nh))) return rc;
  return status;
}

int qexstag_force_solve(qexstag_links *g, double *psi, const double *phi, double m,
                        const qexstag_solver_params *p, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (!psi || !phi) return fail(QEXSTAG_ERR_ARG, "force_solve: null field");
  qexstag_solver_stats st;
  init_stats(&st);
  Timer tm;
  const double2 *dphi;
  double2 *dpsi;
  if ((rc = stage_in(g, kSlotIn0, phi, mem, &dphi))) return rc;
  if ((rc = stage_out_buf(g, kSlotOut0, psi, mem, &dpsi))) return rc;
  int status = force_solve_dev(g, dpsi, dphi, m, p, &st);
  if (status < 0) return status;
  if ((rc = stage_out_finish(g, dpsi, psi, mem))) return rc;
  st.seconds = tm.seconds();
  st.flops = (double)(g->nl * 4 * 72 + 60) * geo_nh(g) * st.iterations;
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

int qexstag_force(qexstag_links *g, double *f, const double *phi, double m,
                  const qexstag_solver_params *p, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_links(g)) || (rc = check_mem(mem)) || (rc = check_params(p))) return rc;
  if (!f || !phi) return fail(QEXSTAG_ERR_ARG, "force: null field");
  const Geom &geo = g->l->g;
  qexstag_solver_stats st;
  init_stats(&st);
  Timer tm;
  const double2 *dphi;
  double2 *df;
  void *ppsi;
  const size_t fb = sizeof(double2) * 3 * (size_t)geo.V;
  if ((rc = stage_in(g, kSlotIn0, phi, mem, &dphi))) return rc;
  if ((rc = force_buf(g, f, mem, &df))) return rc;
  if ((rc = g->ws.get(kSlotIn1, fb, &ppsi))) return rc;
  double2 *psi = (double2 *)ppsi;
  int status = force_solve_dev(g, psi, dphi, m, p, &st);
  if (status < 0) return status;
  if ((rc = ferm_force64(g, df, psi))) return rc;
  if ((rc = force_out(g, df, f, mem))) return rc;
  st.seconds = tm.seconds();
  st.flops = (double)(g->nl * 4 * 72 + 60) * geo.nh * st.iterations;
  finish_stats(&st);
  if (st_out) *st_out = st;
  return status;
}

}  // extern "C"
