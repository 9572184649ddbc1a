// noalloc.cu -- an allocation-free variant of the even-parity Schur operator.
//
// Some callers cannot let a library call cudaMalloc: hosts that hand nearly
// all device memory to their own pool allocator up front (a lattice code
// holding its gauge fields, solver vectors and eigenvectors in one arena),
// so any further cudaMalloc fails, and hosts that cannot accept the
// device-wide synchronisation cudaMalloc and cudaFree may cause in the middle
// of an asynchronous pipeline.  qexstag_stagD2ee_noalloc serves them: it
// computes exactly what qexstag_stagD2ee computes for device fields, but the
// odd-parity temporary of the two half sweeps lives in a file-scope
// __device__ array of fixed size instead of the handle's workspace, and the
// call allocates nothing.
//
// Limits and sharing: the array holds 3 * 65536 double2 (3 MiB), so the
// lattice may have at most 65536 even sites (V <= 131072, e.g. 16^4 or
// 16^3 x 32); larger lattices are rejected.  Every GPU that loads this
// library holds those 3 MiB until the process exits.  All calls on a device
// share the one array and it keeps the last call's contents; the first half
// sweep overwrites every entry the second reads, so nothing needs clearing,
// but two calls that run at the same time on the GPU (different streams, or
// different host threads) race on it.  The first call on each device looks up
// the array's device address (cudaGetSymbolAddress), so make that first
// call before any stream capture.  The address is cached per device until
// qexstag_finalize, which forgets it: a host that resets the device
// (cudaDeviceReset) calls qexstag_finalize first, because after a reset the
// module can load at another address; the next call then looks it up again.
#include <mutex>

#include "lib.cuh"

namespace qs {

int schur64_plain(const qexstag_links_s *gl, int par, VecD r, CVecD x, VecD t, double m2);

constexpr int kNoAllocMaxHalf = 1 << 16;
static __device__ __align__(256) double2 g_noalloc_tmp[3 * kNoAllocMaxHalf];

namespace {
constexpr int kNoAllocDevices = 64;
std::mutex g_noalloc_mutex;
double2 *g_noalloc_ptr[kNoAllocDevices] = {};
}  // namespace

// device address of the array on device dev (looked up once per device,
// with that device current)
static int noalloc_tmp(int dev, double2 **out) {
  if (dev < 0 || dev >= kNoAllocDevices) return fail(QEXSTAG_ERR_ARG, "stagD2ee_noalloc: device out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tmp);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_tmp)");
    g_noalloc_ptr[dev] = (double2 *)p;
  }
  *out = g_noalloc_ptr[dev];
  return QEXSTAG_OK;
}

// forget the cached address on device dev (qexstag_finalize)
void noalloc_forget(int dev) {
  if (dev < 0 || dev >= kNoAllocDevices) return;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  g_noalloc_ptr[dev] = nullptr;
}

}  // namespace qs

extern "C" int qexstag_stagD2ee_noalloc(qexstag_links *g, double *r, const double *x, double m2) {
  using namespace qs;
  if (!g || !g->l || !g->u64) return fail(QEXSTAG_ERR_ARG, "stagD2ee_noalloc: null or destroyed link handle");
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "stagD2ee_noalloc: null field");
  const Geom &geo = g->l->g;
  if (geo.nh > kNoAllocMaxHalf)
    return fail(QEXSTAG_ERR_ARG, "stagD2ee_noalloc: lattice has " + std::to_string(geo.nh) +
                                     " even sites, more than the 65536 its static 3 MiB temporary "
                                     "holds; use qexstag_stagD2ee");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != g->l->device) return fail(QEXSTAG_ERR_STATE, "stagD2ee_noalloc: link handle belongs to another device");
  double2 *t = nullptr;
  int rc = noalloc_tmp(dev, &t);
  if (rc) return rc;
  return schur64_plain(g, 0, block((double2 *)r, geo, 0), block((const double2 *)x, geo, 0),
                       VecD{t, geo.nh}, m2);
}
