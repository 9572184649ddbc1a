// domain.cu -- domain decomposition of the staggered operator and its CG
// along the time direction (scope row F3; QEX's rankGeom split with
// ShiftB boundary exchanges, src/layout/shifts.nim:76-103, 263-294,
// src/layout/qshifts.nim:23-177, src/comms/halo.nim).
//
// Rank r of R holds the time slices [r T, (r+1) T) of the global lattice
// (T = L3 / R, even) as an extended lattice of T + 2h slices: h ghost slices
// below and above, h = 6 for fat+Naik links and 2 for naive links (even, so
// that a site's parity in the extended lattice is its global parity).  With
// ghosts six slices deep the Schur operator's intermediate odd field is
// correct on every slice the second half sweep reads, so one exchange of
// the even input per application suffices and the library's FP64 Schur
// kernels run unchanged on the extended lattice (the values they produce on
// ghost slices are never used).  Reductions run over interior sites only,
// are summed over the domains a process holds in rank order, and then over
// processes.
//
// Neighbours held by the same process (several ranks on one device) are
// exchanged by device-to-device copies; neighbours in other processes by
// NCCL send/receive of the boundary slices into the receiver's ghost slices
// and an NCCL all-reduce of the partial sums.  The exchange runs on a side
// stream while the sweeps that need no ghost run on the library's stream:
// with reach rho (3 with Naik links, 1 without; h = 2 rho) the odd
// intermediate on slices [h+rho, h+T-rho) and the even output on
// [h+2rho, h+T-2rho) read interior slices only; the 2 rho slices at each
// end of both sweeps follow the exchange.
//
// The CG keeps its scalars on the device (the CgState of the one-lattice
// CG): each domain's interior partial sum goes to a slot, one thread adds
// the slots in rank order, NCCL all-reduces that value in place, and the
// next kernel finishes alpha or beta, so an iteration makes no host round
// trip and the host reads the state every few iterations.
//
// Along t, then z: qexstag_domain_create_zt splits the lattice over a grid
// of Rz x Rt ranks (rank = rz + Rz rt), each holding Z = L2 / Rz by T =
// L3 / Rt slabs extended by h ghost rows in z as well.  The exchange fills
// the t ghost slices first (whole slices, z ghost rows included) and then
// the z ghost rows of every slice (t ghost slices included), so the corner
// regions receive the diagonal neighbour's sites by way of the z
// neighbour's t ghosts.  Within a t slice each (z, t) row of L0 L1 / 2 sites
// of a parity is contiguous, so a z face is a pitched 2D copy, packed into a
// contiguous buffer for NCCL.  Both sweeps then run on the whole extended
// slab after the exchange (no overlap); the values they produce on z ghost
// rows are finite and never read, and every sum skips those rows.  A grid
// with Rz = 1 still carries z ghosts and exchanges them with itself.  NCCL is resolved at run time
// from the libnccl.so.2 already loaded in the process (the one torch
// carries) or the system's, so the library does not link a second copy.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "lib.cuh"

namespace qs {

// ---- NCCL through dlsym ----
struct NcclApi {
  bool ok = false;
  ncclResult_t (*getUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*allReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*groupStart)() = nullptr;
  ncclResult_t (*groupEnd)() = nullptr;
  const char *(*errorString)(ncclResult_t) = nullptr;
};

static NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.getUniqueId = (decltype(api.getUniqueId))dlsym(h, "ncclGetUniqueId");
    api.commInitRank = (decltype(api.commInitRank))dlsym(h, "ncclCommInitRank");
    api.commDestroy = (decltype(api.commDestroy))dlsym(h, "ncclCommDestroy");
    api.send = (decltype(api.send))dlsym(h, "ncclSend");
    api.recv = (decltype(api.recv))dlsym(h, "ncclRecv");
    api.allReduce = (decltype(api.allReduce))dlsym(h, "ncclAllReduce");
    api.groupStart = (decltype(api.groupStart))dlsym(h, "ncclGroupStart");
    api.groupEnd = (decltype(api.groupEnd))dlsym(h, "ncclGroupEnd");
    api.errorString = (decltype(api.errorString))dlsym(h, "ncclGetErrorString");
    api.ok = api.getUniqueId && api.commInitRank && api.commDestroy && api.send && api.recv && api.allReduce &&
             api.groupStart && api.groupEnd && api.errorString;
  });
  return api;
}

static int nccl_fail(ncclResult_t r, const char *what) {
  return fail(QEXSTAG_ERR_CUDA, std::string(what) + ": " + (nccl().errorString ? nccl().errorString(r) : "NCCL"));
}
#define QS_NCCL(call)                                       \
  do {                                                      \
    ncclResult_t r_ = (call);                               \
    if (r_ != ncclSuccess) return ::qs::nccl_fail(r_, #call); \
  } while (0)

}  // namespace qs

struct qexstag_domain_s {
  int gdims[4];
  int nranks, rank, nl, h, T;
  int Rz = 1, Rt = 1, rz = 0, rt = 0;  // rank grid (z, t) and this rank's place
  int Z = 0, hz = 0;                // interior z extent and z ghost depth (0: t only)
  qexstag_layout_s *ext = nullptr;  // extended lattice (Z + 2hz rows, T + 2h slices)
  qexstag_links_s *g = nullptr;     // links on the extended lattice
  qexstag_domain_s *up = nullptr, *down = nullptr;    // in-process t neighbours
  qexstag_domain_s *zup = nullptr, *zdown = nullptr;  // in-process z neighbours
  ncclComm_t comm = nullptr;        // inter-process neighbours
  bool hostc = false;               // inter-process through the host communicator hc
  qexstag_host_comm hc{};
  void *hbuf = nullptr;             // pinned staging of host-communicator exchanges
  size_t hbuf_bytes = 0;
  bool connected = false;
  std::vector<qs::Geom> local;      // geometry of the T-slice local lattice
  double *dsum = nullptr;           // device scalars: see DevScalars
  cudaStream_t side = nullptr;      // ghost exchange, overlapped with the interior
  cudaEvent_t fork = nullptr, join = nullptr;
};

namespace qs {

// workspace slots of a domain's link handle
enum DomainSlot {
  kDmIn = kSlotLast + 700, kDmOut, kDmT, kDmFull, kDmX, kDmR, kDmP, kDmAp, kDmSoa, kDmLinks,
  kDmPack,  // four NCCL z-face buffers (send down, send up, receive down, receive up)
  kDmMix    // five compact interior FP64 fields of the mixed-precision solve
};

// layout of a domain's device scalars (dsum): the partial sums of up to
// kMaxSet domains of one call, the combined value, then the CG state
constexpr int kMaxSet = 64;
constexpr int kValOff = kMaxSet;
constexpr int kStateOff = kMaxSet + 8;
constexpr size_t kDevScalarBytes = sizeof(double) * kStateOff + sizeof(CgState);

int write_state(CgState *dst, const CgState &host);
int check_interval(int nh);
int build_low_links(qexstag_links_s *g);
void free_low_links(LowLinks &low);

// sites of one parity in one (z, t) row, and in one t slice of the
// extended lattice
static size_t row_half(const qexstag_domain_s *d) { return (size_t)d->gdims[0] * d->gdims[1] / 2; }
static size_t slice_half(const qexstag_domain_s *d) { return row_half(d) * (size_t)(d->Z + 2 * d->hz); }
static int rank_of(const qexstag_domain_s *d, int rz, int rt) {
  return (rz + d->Rz) % d->Rz + d->Rz * ((rt + d->Rt) % d->Rt);
}

// z faces: rows [row0, row0 + hz) of every t slice of parity block par, for
// components c0 .. c0 + nc - 1, to or from a contiguous buffer
// [nc][Te][hz * P]
__global__ void face_copy_kernel(double2 *field, size_t V, size_t base, size_t pitch, double2 *buf, int nc,
                                 int rows, size_t width, int to_buf) {
  const size_t per = (size_t)rows * width, n = (size_t)nc * per;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / per, rem = i - c * per, s = rem / width, j = rem - s * width;
    const size_t f = c * V + base + s * pitch + j;
    if (to_buf)
      buf[i] = field[f];
    else
      field[f] = buf[i];
  }
}

static int find_in_set(qexstag_domain_s *const *ds, int n, const qexstag_domain_s *d) {
  for (int j = 0; j < n; j++)
    if (ds[j] == d) return j;
  return -1;
}

// pinned staging for the host communicator: four buffers of bytes each
// (send down, send up, receive down, receive up)
static int host_bufs(qexstag_domain_s *d, size_t bytes, char **b) {
  if (d->hbuf_bytes < 4 * bytes) {
    if (d->hbuf) {
      cudaStreamSynchronize(stream());
      cudaStreamSynchronize(d->side);
      cudaFreeHost(d->hbuf);
      d->hbuf = nullptr;
      d->hbuf_bytes = 0;
    }
    if (cudaHostAlloc(&d->hbuf, 4 * bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      d->hbuf = nullptr;
      return fail(QEXSTAG_ERR_ALLOC, "domain: pinned staging for the host communicator failed");
    }
    d->hbuf_bytes = 4 * bytes;
  }
  *b = (char *)d->hbuf;
  return QEXSTAG_OK;
}

// One exchange through the host communicator: receive both ghost faces,
// send both boundary faces (tag: direction of travel), wait.  The faces are
// in host memory already (sdn, sup), the received ones land in rdn, rup.
static int host_swap(qexstag_domain_s *d, int dnr, int upr, const void *sdn, const void *sup, void *rdn, void *rup,
                     size_t bytes, int tag_up, int tag_dn) {
  const qexstag_host_comm &c = d->hc;
  if (c.push_recv(c.ctx, dnr, tag_up, rdn, bytes) || c.push_recv(c.ctx, upr, tag_dn, rup, bytes) ||
      c.push_send(c.ctx, upr, tag_up, sup, bytes) || c.push_send(c.ctx, dnr, tag_dn, sdn, bytes) ||
      c.wait_all(c.ctx))
    return fail(QEXSTAG_ERR_STATE, "domain: the host communicator reported an error");
  return QEXSTAG_OK;
}

// z ghost rows of every t slice of one parity block (after the t ghosts)
static int exchange_z(qexstag_domain_s *const *ds, int n, double2 *const *base, int ncomp, int par,
                      cudaStream_t s) {
  const qexstag_domain_s *d0 = ds[0];
  const size_t P = row_half(d0), pitch = slice_half(d0), width = (size_t)d0->hz * P;
  const int rows = d0->T + 2 * d0->h, Z = d0->Z, hz = d0->hz;
  for (int k = 0; k < n; k++) {
    qexstag_domain_s *d = ds[k];
    const size_t V = (size_t)d->ext->g.V, off = (size_t)par * d->ext->g.nh;
    if (d->hostc) {
      const int upr = rank_of(d, d->rz + 1, d->rt), dnr = rank_of(d, d->rz - 1, d->rt);
      for (int c0 = 0; c0 < ncomp; c0 += 3) {
        const int nc = std::min(3, ncomp - c0);
        const size_t face = (size_t)nc * rows * width, bytes = face * sizeof(double2);
        void *pb;
        char *hb;
        int rc = d->g->ws.get(kDmPack, sizeof(double2) * 4 * (size_t)3 * rows * width, &pb);
        if (rc || (rc = host_bufs(d, bytes, &hb))) return rc;
        double2 *sdn = (double2 *)pb, *sup = sdn + face, *rdn = sup + face, *rup = rdn + face;
        double2 *f = base[k] + (size_t)c0 * V;
        const int grid = grid_for((long)face);
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)hz * P, pitch, sdn, nc, rows, width, 1);
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)Z * P, pitch, sup, nc, rows, width, 1);
        note_launch(2);
        QS_LAUNCH_CHECK();
        QS_CUDA(cudaMemcpyAsync(hb, sdn, 2 * bytes, cudaMemcpyDeviceToHost, s));  // sdn, sup are adjacent
        QS_CUDA(cudaStreamSynchronize(s));
        if ((rc = host_swap(d, dnr, upr, hb, hb + bytes, hb + 2 * bytes, hb + 3 * bytes, bytes, 2, 3))) return rc;
        QS_CUDA(cudaMemcpyAsync(rdn, hb + 2 * bytes, 2 * bytes, cudaMemcpyHostToDevice, s));  // rdn, rup adjacent
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off, pitch, rdn, nc, rows, width, 0);
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)(hz + Z) * P, pitch, rup, nc, rows, width, 0);
        note_launch(2);
        QS_LAUNCH_CHECK();
        QS_CUDA(cudaStreamSynchronize(s));
      }
    } else if (d->comm) {
      const int upr = rank_of(d, d->rz + 1, d->rt), dnr = rank_of(d, d->rz - 1, d->rt);
      for (int c0 = 0; c0 < ncomp; c0 += 3) {
        const int nc = std::min(3, ncomp - c0);
        const size_t face = (size_t)nc * rows * width;
        void *pb;
        int rc = d->g->ws.get(kDmPack, sizeof(double2) * 4 * (size_t)3 * rows * width, &pb);
        if (rc) return rc;
        double2 *sdn = (double2 *)pb, *sup = sdn + face, *rdn = sup + face, *rup = rdn + face;
        double2 *f = base[k] + (size_t)c0 * V;
        const int grid = grid_for((long)face);
        // my lowest interior rows go down, my highest up
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)hz * P, pitch, sdn, nc, rows, width, 1);
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)Z * P, pitch, sup, nc, rows, width, 1);
        note_launch(2);
        QS_LAUNCH_CHECK();
        QS_NCCL(nccl().groupStart());
        QS_NCCL(nccl().send(sdn, 2 * face, ncclDouble, dnr, d->comm, s));
        QS_NCCL(nccl().recv(rup, 2 * face, ncclDouble, upr, d->comm, s));
        QS_NCCL(nccl().send(sup, 2 * face, ncclDouble, upr, d->comm, s));
        QS_NCCL(nccl().recv(rdn, 2 * face, ncclDouble, dnr, d->comm, s));
        QS_NCCL(nccl().groupEnd());
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off, pitch, rdn, nc, rows, width, 0);
        face_copy_kernel<<<grid, kBlock, 0, s>>>(f, V, off + (size_t)(hz + Z) * P, pitch, rup, nc, rows, width, 0);
        note_launch(2);
        QS_LAUNCH_CHECK();
      }
    } else {
      const int ku = find_in_set(ds, n, d->zup), kd = find_in_set(ds, n, d->zdown);
      if (ku < 0 || kd < 0) return fail(QEXSTAG_ERR_STATE, "domain: a z neighbour is not in the call's domain set");
      for (int c = 0; c < ncomp; c++) {
        double2 *f = base[k] + (size_t)c * V + off;
        const double2 *fd = base[kd] + (size_t)c * V + off;
        const double2 *fu = base[ku] + (size_t)c * V + off;
        // lower ghost rows <- the z-down neighbour's highest interior rows, upper <- z-up's lowest
        QS_CUDA(cudaMemcpy2DAsync(f, pitch * sizeof(double2), fd + (size_t)Z * P, pitch * sizeof(double2),
                                  width * sizeof(double2), rows, cudaMemcpyDeviceToDevice, s));
        QS_CUDA(cudaMemcpy2DAsync(f + (size_t)(hz + Z) * P, pitch * sizeof(double2), fu + (size_t)hz * P,
                                  pitch * sizeof(double2), width * sizeof(double2), rows, cudaMemcpyDeviceToDevice,
                                  s));
      }
    }
  }
  return QEXSTAG_OK;
}

// one parity block's ghost exchange of ncomp component arrays, each with
// stride V_ext, of the fields at base[k] of each domain of the set: t ghost
// slices, then (domains split along z) the z ghost rows of every slice
static int exchange(qexstag_domain_s *const *ds, int n, double2 *const *base, int ncomp, int par,
                    cudaStream_t s) {
  const size_t sh = slice_half(ds[0]);
  for (int k = 0; k < n; k++) {
    qexstag_domain_s *d = ds[k];
    const size_t V = (size_t)d->ext->g.V, nh = (size_t)d->ext->g.nh;
    const size_t cnt = d->h * sh;  // sites per face per component
    if (d->hostc) {
      // faces of every component through pinned host memory, [ncomp][cnt]
      const int upr = rank_of(d, d->rz, d->rt + 1), dnr = rank_of(d, d->rz, d->rt - 1);
      const size_t per = cnt * sizeof(double2), bytes = per * ncomp;
      char *hb;
      int rc = host_bufs(d, bytes, &hb);
      if (rc) return rc;
      char *sdn = hb, *sup = hb + bytes, *rdn = hb + 2 * bytes, *rup = hb + 3 * bytes;
      for (int c = 0; c < ncomp; c++) {
        const double2 *f = base[k] + (size_t)c * V + (size_t)par * nh;
        QS_CUDA(cudaMemcpyAsync(sup + c * per, f + (size_t)d->T * sh, per, cudaMemcpyDeviceToHost, s));
        QS_CUDA(cudaMemcpyAsync(sdn + c * per, f + (size_t)d->h * sh, per, cudaMemcpyDeviceToHost, s));
      }
      QS_CUDA(cudaStreamSynchronize(s));
      if ((rc = host_swap(d, dnr, upr, sdn, sup, rdn, rup, bytes, 0, 1))) return rc;
      for (int c = 0; c < ncomp; c++) {
        double2 *f = base[k] + (size_t)c * V + (size_t)par * nh;
        QS_CUDA(cudaMemcpyAsync(f, rdn + c * per, per, cudaMemcpyHostToDevice, s));
        QS_CUDA(cudaMemcpyAsync(f + (size_t)(d->h + d->T) * sh, rup + c * per, per, cudaMemcpyHostToDevice, s));
      }
      // the staging is reused by the next exchange: let these copies finish
      QS_CUDA(cudaStreamSynchronize(s));
    } else if (d->comm) {
      QS_NCCL(nccl().groupStart());
      const int upr = rank_of(d, d->rz, d->rt + 1), dnr = rank_of(d, d->rz, d->rt - 1);
      for (int c = 0; c < ncomp; c++) {
        double2 *f = base[k] + (size_t)c * V + (size_t)par * nh;
        // my top interior slices -> up's lower ghosts; my bottom -> down's upper
        QS_NCCL(nccl().send(f + (size_t)d->T * sh, 2 * cnt, ncclDouble, upr, d->comm, s));
        QS_NCCL(nccl().recv(f, 2 * cnt, ncclDouble, dnr, d->comm, s));
        QS_NCCL(nccl().send(f + (size_t)d->h * sh, 2 * cnt, ncclDouble, dnr, d->comm, s));
        QS_NCCL(nccl().recv(f + (size_t)(d->h + d->T) * sh, 2 * cnt, ncclDouble, upr, d->comm, s));
      }
      QS_NCCL(nccl().groupEnd());
    } else {
      // pull from the in-process neighbours
      const int ku = find_in_set(ds, n, d->up), kd = find_in_set(ds, n, d->down);
      if (ku < 0 || kd < 0) return fail(QEXSTAG_ERR_STATE, "domain: a neighbour is not in the call's domain set");
      for (int c = 0; c < ncomp; c++) {
        double2 *f = base[k] + (size_t)c * V + (size_t)par * nh;
        const double2 *fd = base[kd] + (size_t)c * V + (size_t)par * nh;
        const double2 *fu = base[ku] + (size_t)c * V + (size_t)par * nh;
        QS_CUDA(cudaMemcpyAsync(f, fd + (size_t)d->down->T * sh, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        QS_CUDA(cudaMemcpyAsync(f + (size_t)(d->h + d->T) * sh, fu + (size_t)d->up->h * sh, cnt * sizeof(double2),
                                cudaMemcpyDeviceToDevice, s));
      }
    }
  }
  if (ds[0]->hz > 0) return exchange_z(ds, n, base, ncomp, par, s);
  return QEXSTAG_OK;
}

// sum of the n domains' device scalars (rank order), then over processes
static int allreduce_sum(qexstag_domain_s *const *ds, int n, const double *vals, double *out) {
  double s = 0;
  for (int k = 0; k < n; k++) s += vals[k];
  qexstag_domain_s *d = ds[0];
  if (d->hostc) {
    if (d->hc.all_reduce_sum(d->hc.ctx, &s, 1))
      return fail(QEXSTAG_ERR_STATE, "domain: the host communicator's sum reported an error");
  } else if (d->comm) {
    QS_CUDA(cudaMemcpyAsync(d->dsum, &s, sizeof(double), cudaMemcpyHostToDevice, stream()));
    QS_NCCL(nccl().allReduce(d->dsum, d->dsum, 1, ncclDouble, ncclSum, d->comm, stream()));
    QS_CUDA(cudaMemcpyAsync(&s, d->dsum, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));
  }
  *out = s;
  return QEXSTAG_OK;
}

// local V=1 site order (Z x T slab) <-> extended lattice (z + hz, t + h)
__global__ void local_to_ext_kernel(Geom loc, Geom ext, int hz, int h, const double2 *in, size_t ins,
                                    double2 *out, size_t outs, int ncomp, int to_ext) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < loc.V; i += gridDim.x * blockDim.x) {
    const int par = i >= loc.nh ? 1 : 0;
    int x[4], lex;
    site_coords(loc, par, i - par * loc.nh, x, lex);
    const int elex = x[0] + ext.L[0] * (x[1] + ext.L[1] * (x[2] + hz + ext.L[2] * (x[3] + h)));
    const int j = (elex >> 1) + par * ext.nh;  // same parity (hz, h even)
    for (int c = 0; c < ncomp; c++) {
      if (to_ext)
        out[(size_t)c * outs + j] = in[(size_t)c * ins + i];
      else
        out[(size_t)c * outs + i] = in[(size_t)c * ins + j];
    }
  }
}

__global__ void unit_links_kernel(size_t n, double2 *u) {
  // n = nlinks * V sites of links; element e of link l at (l * 9 + e) * V + s
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 9 * n; i += (size_t)gridDim.x * blockDim.x)
    u[i] = make_double2(0.0, 0.0);
}
__global__ void unit_diag_kernel(int nl, int V, double2 *u) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V; s += gridDim.x * blockDim.x)
    for (int l = 0; l < nl; l++)
      for (int e = 0; e < 9; e += 4) u[((size_t)l * 9 + e) * V + s] = make_double2(1.0, 0.0);
}

static int convert(qexstag_domain_s *d, const double2 *in, size_t ins, double2 *out, size_t outs, int ncomp,
                   bool to_ext) {
  const Geom &loc = d->local[0];
  local_to_ext_kernel<<<grid_for(loc.V), kBlock, 0, stream()>>>(loc, d->ext->g, d->hz, d->h, in, ins, out, outs,
                                                                ncomp, to_ext ? 1 : 0);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

static int check_set(qexstag_domain_s *const *ds, int n) {
  if (!ds || n < 1) return fail(QEXSTAG_ERR_ARG, "domain: empty domain set");
  for (int k = 0; k < n; k++) {
    if (!ds[k]) return fail(QEXSTAG_ERR_ARG, "domain: null domain");
    if (!ds[k]->connected) return fail(QEXSTAG_ERR_STATE, "domain: not connected to its neighbours");
    if (ds[k]->nl != ds[0]->nl || std::memcmp(ds[k]->gdims, ds[0]->gdims, sizeof ds[0]->gdims) ||
        ds[k]->nranks != ds[0]->nranks || ds[k]->Rz != ds[0]->Rz || ds[k]->hz != ds[0]->hz)
      return fail(QEXSTAG_ERR_ARG, "domain: domains of different lattices in one call");
    if ((ds[k]->comm != nullptr) != (ds[0]->comm != nullptr) || ds[k]->hostc != ds[0]->hostc)
      return fail(QEXSTAG_ERR_ARG, "domain: domains with different connections in one call");
  }
  if (n > kMaxSet) return fail(QEXSTAG_ERR_ARG, "domain: more than 64 domains in one call");
  if ((ds[0]->comm || ds[0]->hostc) && n > 1)
    return fail(QEXSTAG_ERR_ARG, "domain: one NCCL- or host-connected domain per call");
  return runtime_ready();
}

// device copy (extended layout) of each domain's local full-lattice colour
// vector; host fields [Vloc][3] or device [3][Vloc]
struct ExtVec {
  std::vector<double2 *> p;
};

static int vec_slot_get(qexstag_domain_s *d, int slot, double2 **out) {
  void *q;
  int rc = d->g->ws.get(slot, sizeof(double2) * 3 * (size_t)d->ext->g.V, &q);
  if (rc) return rc;
  *out = (double2 *)q;
  return QEXSTAG_OK;
}

static int vec_in(qexstag_domain_s *d, int slot, const double *x, int mem, double2 **ext) {
  int rc;
  if ((rc = vec_slot_get(d, slot, ext))) return rc;
  QS_CUDA(cudaMemsetAsync(*ext, 0, sizeof(double2) * 3 * (size_t)d->ext->g.V, stream()));
  const size_t Vl = (size_t)d->local[0].V;
  const double2 *src = (const double2 *)x;
  if (mem == QEXSTAG_MEM_HOST) {
    void *aos, *soa;
    if ((rc = d->g->ws.get(kSlotAos, sizeof(double2) * 3 * Vl, &aos)) ||
        (rc = d->g->ws.get(kDmSoa, sizeof(double2) * 3 * Vl, &soa)))
      return rc;
    QS_CUDA(cudaMemcpyAsync(aos, x, sizeof(double2) * 3 * Vl, cudaMemcpyHostToDevice, stream()));
    if ((rc = aos_to_soa((const double *)aos, (double2 *)soa, (int)Vl, (int)Vl, 3))) return rc;
    src = (const double2 *)soa;
  }
  return convert(d, src, Vl, *ext, d->ext->g.V, 3, true);
}

static int vec_out(qexstag_domain_s *d, const double2 *ext, double *x, int mem) {
  const size_t Vl = (size_t)d->local[0].V;
  int rc;
  if (mem == QEXSTAG_MEM_DEVICE) return convert(d, ext, d->ext->g.V, (double2 *)x, Vl, 3, false);
  void *aos, *soa;
  if ((rc = d->g->ws.get(kSlotAos, sizeof(double2) * 3 * Vl, &aos)) ||
      (rc = d->g->ws.get(kDmSoa, sizeof(double2) * 3 * Vl, &soa)))
    return rc;
  if ((rc = convert(d, ext, d->ext->g.V, (double2 *)soa, Vl, 3, false)) ||
      (rc = soa_to_aos((const double2 *)soa, (double *)aos, (int)Vl, (int)Vl, 3)))
    return rc;
  QS_CUDA(cudaMemcpyAsync(x, aos, sizeof(double2) * 3 * Vl, cudaMemcpyDeviceToHost, stream()));
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

// interior even block of an extended field
static VecD interior(qexstag_domain_s *d, double2 *f) {
  return VecD{f + d->h * slice_half(d), d->ext->g.V};
}
static int interior_n(qexstag_domain_s *d) { return (int)(d->T * slice_half(d)); }

// r = stagD2ee(m2) x on every domain (even interior sites; t is the odd
// block of the intermediate).  The ghost exchange of x runs on the side
// stream while the sweeps that read interior slices only run on the
// library's stream; the slices next to the ghosts follow the exchange.
// Skipped once *done is set (the exchange still runs, unread).
static int schur_set(qexstag_domain_s *const *ds, int n, double2 *const *r, double2 *const *x, double2 *const *t,
                     double m2, const int *done = nullptr) {
  int rc;
  qexstag_domain_s *d0 = ds[0];
  const int sh = (int)slice_half(d0), h = d0->h, T = d0->T;
  const int rho = h / 2;                 // reach of the longest hop
  // some slices need no ghost at all (t splits only: with z ghosts every
  // slice has ghost rows)
  const bool overlap = d0->hz == 0 && T > 4 * rho;
  QS_CUDA(cudaEventRecord(d0->fork, stream()));
  QS_CUDA(cudaStreamWaitEvent(d0->side, d0->fork, 0));
  if ((rc = exchange(ds, n, x, 3, 0, d0->side))) return rc;
  QS_CUDA(cudaEventRecord(d0->join, d0->side));
  for (int k = 0; overlap && k < n; k++) {
    const Geom &g = ds[k]->ext->g;
    const CVecD xe{x[k], g.V}, te{t[k] + g.nh, g.V};
    // t = (2D)_oe x on [h+rho, h+T-rho), r = 4 m2 x - (2D)_eo t on [h+2rho, h+T-2rho)
    if ((rc = dslash64_ranges(ds[k]->g, 1, VecD{t[k] + g.nh, g.V}, xe, CVecD{nullptr, 0}, 0.0, 1.0, +1,
                              (h + rho) * sh, (h + T - rho) * sh, 0, 0, done)) ||
        (rc = dslash64_ranges(ds[k]->g, 0, VecD{r[k], g.V}, te, xe, 4.0 * m2, 1.0, -1, (h + 2 * rho) * sh,
                              (h + T - 2 * rho) * sh, 0, 0, done)))
      return rc;
  }
  QS_CUDA(cudaStreamWaitEvent(stream(), d0->join, 0));
  for (int k = 0; k < n; k++) {
    const Geom &g = ds[k]->ext->g;
    const CVecD xe{x[k], g.V}, te{t[k] + g.nh, g.V};
    if (overlap) {
      rc = dslash64_ranges(ds[k]->g, 1, VecD{t[k] + g.nh, g.V}, xe, CVecD{nullptr, 0}, 0.0, 1.0, +1,
                           (h - rho) * sh, (h + rho) * sh, (h + T - rho) * sh, (h + T + rho) * sh, done);
      if (!rc)
        rc = dslash64_ranges(ds[k]->g, 0, VecD{r[k], g.V}, te, xe, 4.0 * m2, 1.0, -1, h * sh, (h + 2 * rho) * sh,
                             (h + T - 2 * rho) * sh, (h + T) * sh, done);
    } else if (d0->hz > 0) {
      // z splits: the intermediate on rows [hz-rho, hz+Z+rho) of slices
      // [h-rho, h+T+rho), the output on the interior rows of [h, h+T)
      const int P = (int)row_half(d0), hz = d0->hz, Z = d0->Z;
      rc = dslash64_rows(ds[k]->g, 1, VecD{t[k] + g.nh, g.V}, xe, CVecD{nullptr, 0}, 0.0, 1.0, +1,
                         (h - rho) * sh + (hz - rho) * P, T + 2 * rho, (Z + 2 * rho) * P, sh, done);
      if (!rc)
        rc = dslash64_rows(ds[k]->g, 0, VecD{r[k], g.V}, te, xe, 4.0 * m2, 1.0, -1, h * sh + hz * P, T, Z * P, sh,
                           done);
    } else {
      rc = dslash64_ranges(ds[k]->g, 1, VecD{t[k] + g.nh, g.V}, xe, CVecD{nullptr, 0}, 0.0, 1.0, +1,
                           (h - rho) * sh, (h + T + rho) * sh, 0, 0, done);
      if (!rc)
        rc = dslash64_ranges(ds[k]->g, 0, VecD{r[k], g.V}, te, xe, 4.0 * m2, 1.0, -1, h * sh, (h + T) * sh, 0, 0,
                             done);
    }
    if (rc) return rc;
  }
  return QEXSTAG_OK;
}

// ---- device-resident CG over the domains ----

// which sites of an interior block (t slices [h, h+T), all rows) are not z
// ghosts: row i / P of the block lies at z = row mod Ze; hz = 0 keeps all
struct Rows {
  int P, Ze, hz, Z;
};
static Rows rows_of(const qexstag_domain_s *d) {
  return Rows{(int)row_half(d), d->Z + 2 * d->hz, d->hz, d->Z};
}
__device__ __forceinline__ bool in_z(const Rows &w, int i) {
  if (w.hz == 0) return true;
  const int z = (i / w.P) % w.Ze;
  return z >= w.hz && z < w.hz + w.Z;
}

__global__ void __launch_bounds__(kBlock)
    dm_p_kernel(const double2 *__restrict__ r, double2 *__restrict__ p, int stride, int n, const CgState *st) {
  if (st->done) return;
  const bool first = (st->itn == 0);
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 rv = r[(size_t)c * stride + i];
      if (first) {
        p[(size_t)c * stride + i] = rv;
      } else {
        const double2 pv = p[(size_t)c * stride + i];
        p[(size_t)c * stride + i] = make_double2(fma(beta, pv.x, rv.x), fma(beta, pv.y, rv.y));
      }
    }
  }
}

// Re <a, b> over one domain's interior into *slot (st may be null)
__global__ void __launch_bounds__(kBlock)
    dm_dot_kernel(const double2 *__restrict__ a, const double2 *__restrict__ b, int stride, int n, Rows w,
                  const CgState *st, double *slot, double *partials, unsigned *ticket) {
  if (st != nullptr && st->done) return;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!in_z(w, i)) continue;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 u = a[(size_t)c * stride + i], v = b[(size_t)c * stride + i];
      s = fma(u.x, v.x, s);
      s = fma(u.y, v.y, s);
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) *slot = o[0];
}

// x += alpha p, r -= alpha Ap on one domain's interior; |r|^2 into *slot
__global__ void __launch_bounds__(kBlock)
    dm_xr_kernel(double2 *__restrict__ x, double2 *__restrict__ r, const double2 *__restrict__ p,
                 const double2 *__restrict__ ap, int stride, int n, Rows w, const CgState *st, double *slot,
                 double *partials, unsigned *ticket) {
  if (st->done) return;
  const double alpha = st->alpha;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool keep = in_z(w, i);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const size_t o = (size_t)c * stride + i;
      const double2 pv = p[o], av = ap[o];
      double2 xv = x[o], rv = r[o];
      xv.x = fma(alpha, pv.x, xv.x);
      xv.y = fma(alpha, pv.y, xv.y);
      rv.x = fma(-alpha, av.x, rv.x);
      rv.y = fma(-alpha, av.y, rv.y);
      x[o] = xv;
      r[o] = rv;
      if (keep) {
        s = fma(rv.x, rv.x, s);
        s = fma(rv.y, rv.y, s);
      }
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) *slot = o[0];
}

// One thread: the n slots added in rank order into *val (n = 0: *val as
// the all-reduce left it), then what = 1: pAp, alpha = rz/pAp, itn += 1;
// what = 2: r2, beta = r2/rz, done (cg.nim:213-240).
__global__ void dm_scalar_kernel(const double *slots, int n, double *val, CgState *st, int what) {
  if (st->done) return;
  double s;
  if (n > 0) {
    s = 0.0;
    for (int k = 0; k < n; k++) s += slots[k];
    *val = s;
  } else {
    s = *val;
  }
  if (what == 1) {
    st->pAp = s;
    st->alpha = st->rz / s;
    st->itn += 1;
  } else if (what == 2) {
    st->r2 = s;
    st->beta = s / st->rz;
    st->rz = s;
    if (isnan(s)) st->nan = 1;
    st->done = (!(st->itn < st->maxits && s > st->r2stop) || st->nan) ? 1 : 0;
  }
}

static int finish_scalar(qexstag_domain_s *const *ds, int n, CgState *st, int what) {
  double *slots = ds[0]->dsum, *val = ds[0]->dsum + kValOff;
  if (ds[0]->hostc) {
    // through the host: this process's value out, the sum over processes in
    double *h = host_results();
    dm_scalar_kernel<<<1, 1, 0, stream()>>>(slots, n, val, st, 0);
    note_launch();
    QS_LAUNCH_CHECK();
    QS_CUDA(cudaMemcpyAsync(h, val, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));
    double v = h[0];
    if (ds[0]->hc.all_reduce_sum(ds[0]->hc.ctx, &v, 1))
      return fail(QEXSTAG_ERR_STATE, "domain: the host communicator's sum reported an error");
    h[0] = v;
    QS_CUDA(cudaMemcpyAsync(val, h, sizeof(double), cudaMemcpyHostToDevice, stream()));
    dm_scalar_kernel<<<1, 1, 0, stream()>>>(nullptr, 0, val, st, what);
    note_launch();
    // h is reused by the next call: the copy must have read it
    QS_CUDA(cudaStreamSynchronize(stream()));
  } else if (ds[0]->comm) {
    dm_scalar_kernel<<<1, 1, 0, stream()>>>(slots, n, val, st, 0);
    QS_NCCL(nccl().allReduce(val, val, 1, ncclDouble, ncclSum, ds[0]->comm, stream()));
    dm_scalar_kernel<<<1, 1, 0, stream()>>>(nullptr, 0, val, st, what);
    note_launch(2);
  } else {
    dm_scalar_kernel<<<1, 1, 0, stream()>>>(slots, n, val, st, what);
    note_launch();
  }
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// Re <a, b> (or |a|^2) over the interiors of the set, summed in rank order
// and over processes; z ghost rows left out
static int dot_set(qexstag_domain_s *const *ds, int n, double2 *const *a, double2 *const *b, double *out) {
  std::vector<double> v(n);
  int rc;
  for (int k = 0; k < n; k++) {
    const VecD ia = interior(ds[k], a[k]), ib = interior(ds[k], b[k]);
    if (ds[k]->hz > 0) {
      const int ni = interior_n(ds[k]);
      dm_dot_kernel<<<std::min(grid_for(ni), kMaxRedBlocks), kBlock, 0, stream()>>>(
          ia.p, ib.p, ia.stride, ni, rows_of(ds[k]), nullptr, ds[0]->dsum + k, red_partials(), red_tickets());
      note_launch();
      QS_LAUNCH_CHECK();
      QS_CUDA(cudaMemcpyAsync(&v[k], ds[0]->dsum + k, sizeof(double), cudaMemcpyDeviceToHost, stream()));
      QS_CUDA(cudaStreamSynchronize(stream()));
      rc = QEXSTAG_OK;
    } else if (a == b) {
      rc = vnorm2(cv(ia), interior_n(ds[k]), &v[k]);
    } else {
      rc = vredot(cv(ia), cv(ib), interior_n(ds[k]), &v[k]);
    }
    if (rc) return rc;
  }
  return allreduce_sum(ds, n, v.data(), out);
}

// one CG iteration (cg.nim:174-240, cpNone) enqueued without a host sync
static int cg_iteration(qexstag_domain_s *const *ds, int n, double2 *const *xv, double2 *const *rv,
                        double2 *const *pv, double2 *const *ap, double2 *const *tv, double m2, CgState *st) {
  int rc;
  for (int k = 0; k < n; k++) {
    const int ni = interior_n(ds[k]);
    const VecD r = interior(ds[k], rv[k]), p = interior(ds[k], pv[k]);
    dm_p_kernel<<<grid_for(ni), kBlock, 0, stream()>>>(r.p, p.p, p.stride, ni, st);
  }
  note_launch(n);
  QS_LAUNCH_CHECK();
  if ((rc = schur_set(ds, n, ap, pv, tv, m2, &st->done))) return rc;
  for (int k = 0; k < n; k++) {
    const int ni = interior_n(ds[k]);
    const VecD p = interior(ds[k], pv[k]), a = interior(ds[k], ap[k]);
    dm_dot_kernel<<<std::min(grid_for(ni), kMaxRedBlocks), kBlock, 0, stream()>>>(
        p.p, a.p, p.stride, ni, rows_of(ds[k]), st, ds[0]->dsum + k, red_partials(), red_tickets());
  }
  note_launch(n);
  QS_LAUNCH_CHECK();
  if ((rc = finish_scalar(ds, n, st, 1))) return rc;
  for (int k = 0; k < n; k++) {
    const int ni = interior_n(ds[k]);
    const VecD x = interior(ds[k], xv[k]), r = interior(ds[k], rv[k]), p = interior(ds[k], pv[k]),
               a = interior(ds[k], ap[k]);
    dm_xr_kernel<<<std::min(grid_for(ni), kMaxRedBlocks), kBlock, 0, stream()>>>(
        x.p, r.p, p.p, a.p, p.stride, ni, rows_of(ds[k]), st, ds[0]->dsum + k, red_partials(), red_tickets());
  }
  note_launch(n);
  QS_LAUNCH_CHECK();
  return finish_scalar(ds, n, st, 2);
}

// ---- the mixed-precision solve on one domain per process ----

struct MixedCtx {
  qexstag_domain_s *d;
  double2 *xe, *ae, *te;  // FP64 extended fields for the reliable updates' Schur operator
  double m2;
};

static int mx_exchange_even(void *ctx, void *field) {
  qexstag_domain_s *d = ((MixedCtx *)ctx)->d;
  double2 *f = (double2 *)field;  // 16 bytes per site: one double2 component
  return exchange(&d, 1, &f, 1, 0, stream());
}

static int mx_allreduce(void *ctx, double *dev, int n) {
  qexstag_domain_s *d = ((MixedCtx *)ctx)->d;
  if (d->hostc) {
    double *h = host_results();
    QS_CUDA(cudaMemcpyAsync(h, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));
    double v[4];
    std::memcpy(v, h, sizeof(double) * n);
    if (d->hc.all_reduce_sum(d->hc.ctx, v, n))
      return fail(QEXSTAG_ERR_STATE, "domain: the host communicator's sum reported an error");
    std::memcpy(h, v, sizeof(double) * n);
    QS_CUDA(cudaMemcpyAsync(dev, h, sizeof(double) * n, cudaMemcpyHostToDevice, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));  // h is reused by the next call
  } else if (d->comm) {
    QS_NCCL(nccl().allReduce(dev, dev, n, ncclDouble, ncclSum, d->comm, stream()));
  }
  return QEXSTAG_OK;
}

static int mx_schur64(void *ctx, const double2 *x, double2 *ax) {
  MixedCtx *c = (MixedCtx *)ctx;
  qexstag_domain_s *d = c->d;
  const int ni = interior_n(d);
  int rc;
  if ((rc = vcopy(interior(d, c->xe), CVecD{x, ni}, ni))) return rc;
  if ((rc = schur_set(&d, 1, &c->ae, &c->xe, &c->te, c->m2))) return rc;
  return vcopy(VecD{ax, ni}, cv(interior(d, c->ae)), ni);
}

// FP64 defect correction (stagSolve.nim:330-421) around the 16-bit
// reliable-update CG of cg_mixed_domain; bv: the source on the extended
// lattice, xv: receives the solution's interior even sites.
static int solve_mixed_domain(qexstag_domain_s *d, double2 *bv, double2 *xv, double2 *ae, double2 *te, double m,
                              const qexstag_solver_params *p, qexstag_solver_stats *st, double *r2_out) {
  const int ni = interior_n(d);
  const size_t vb = sizeof(double2) * 3 * (size_t)ni;
  void *pb, *px, *prho, *py, *pax;
  int rc;
  Workspace &ws = d->g->ws;
  if ((rc = ws.get(kDmMix + 0, vb, &pb)) || (rc = ws.get(kDmMix + 1, vb, &px)) || (rc = ws.get(kDmMix + 2, vb, &prho)) ||
      (rc = ws.get(kDmMix + 3, vb, &py)) || (rc = ws.get(kDmMix + 4, vb, &pax)))
    return rc;
  double2 *b = (double2 *)pb, *x = (double2 *)px, *rho = (double2 *)prho, *y = (double2 *)py, *ax = (double2 *)pax;
  const double m2 = m * m;
  MixedCtx ctx{d, xv, ae, te, m2};
  const size_t eb = sizeof(double2) * 3 * (size_t)d->ext->g.V;
  QS_CUDA(cudaMemsetAsync(xv, 0, eb, stream()));
  MxDomain D;
  D.ctx = &ctx;
  D.exchange_even = mx_exchange_even;
  D.allreduce = mx_allreduce;
  D.schur64 = mx_schur64;
  D.g = d->g;
  const int sh = (int)slice_half(d), rho_hop = d->h / 2;
  D.even_lo = d->h * sh;
  D.n = ni;
  D.odd_lo = (d->h - rho_hop) * sh;
  D.odd_hi = (d->h + d->T + rho_hop) * sh;
  if ((rc = vcopy(VecD{b, ni}, cv(interior(d, bv)), ni)) || (rc = vcopy(VecD{rho, ni}, CVecD{b, ni}, ni)) ||
      (rc = vzero(VecD{x, ni}, ni)))
    return rc;
  double b2l = 0, b2 = 0;
  if ((rc = vnorm2(CVecD{b, ni}, ni, &b2l)) || (rc = allreduce_sum(&d, 1, &b2l, &b2))) return rc;
  if (!std::isfinite(b2)) return fail(QEXSTAG_ERR_NAN, "domain_solveEE: source is not finite");
  double r2 = b2, r2prev = INFINITY;
  const double r2stop = p->r2req * b2;
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  const double delta = p->delta > 0 ? p->delta : 0.3;
  while (r2 > r2stop && r2 < r2prev) {
    r2prev = r2;
    const int mx = maxits - st->iterations;
    if (mx <= 0) break;
    CgOut o{};
    int rel = 0;
    if ((rc = cg_mixed_domain(D, m2, rho, y, r2stop / r2, mx, delta, &o, &rel))) return rc;
    st->iterations += o.iterations;
    st->reliable_updates += rel;
    st->outer_iterations += 1;
    double r2l = 0;
    if ((rc = vaxpy(VecD{x, ni}, 1.0, CVecD{y, ni}, ni)) || (rc = mx_schur64(&ctx, x, ax)) ||
        (rc = vsub(VecD{rho, ni}, CVecD{b, ni}, CVecD{ax, ni}, ni)) || (rc = vnorm2(CVecD{rho, ni}, ni, &r2l)) ||
        (rc = allreduce_sum(&d, 1, &r2l, &r2)))
      return rc;
    if (std::isnan(r2)) return fail(QEXSTAG_ERR_NAN, "domain_solveEE: NaN residual");
  }
  // the solution into the extended field's interior (odd sites and ghosts zero)
  QS_CUDA(cudaMemsetAsync(xv, 0, eb, stream()));
  if ((rc = vcopy(interior(d, xv), CVecD{x, ni}, ni))) return rc;
  *r2_out = r2;
  return QEXSTAG_OK;
}

}  // namespace qs

using namespace qs;

extern "C" {

// Rz x Rt ranks (rank = rz + Rz rt); zghost: z ghost rows (qexstag_domain_create_zt)
static int domain_create(const int global_dims[4], int Rz, int Rt, int rank, int nlinks, bool zghost,
                         qexstag_domain **out) {
  if (!global_dims || !out) return fail(QEXSTAG_ERR_ARG, "domain_create: null argument");
  if (nlinks != 4 && nlinks != 8) return fail(QEXSTAG_ERR_ARG, "domain_create: nlinks must be 4 or 8");
  const int nranks = Rz * Rt;
  if (Rz < 1 || Rt < 1 || rank < 0 || rank >= nranks) return fail(QEXSTAG_ERR_ARG, "domain_create: bad rank");
  const int h = nlinks == 8 ? 6 : 2;
  if (global_dims[3] % Rt) return fail(QEXSTAG_ERR_ARG, "domain_create: L3 is not a multiple of the t ranks");
  if (global_dims[2] % Rz) return fail(QEXSTAG_ERR_ARG, "domain_create: L2 is not a multiple of the z ranks");
  const int T = global_dims[3] / Rt, Z = global_dims[2] / Rz;
  if (T % 2 || T < h || T < 4)
    return fail(QEXSTAG_ERR_ARG, "domain_create: slab thickness must be even, at least 4 and at least the ghost "
                                 "depth (6 fat+Naik, 2 naive)");
  if (zghost && (Z % 2 || Z < h || Z < 4))
    return fail(QEXSTAG_ERR_ARG, "domain_create: the z extent of a rank must be even, at least 4 and at least the "
                                 "ghost depth (6 fat+Naik, 2 naive)");
  int rc = runtime_ready();
  if (rc) return rc;
  qexstag_domain_s *d = new (std::nothrow) qexstag_domain_s;
  if (!d) return fail(QEXSTAG_ERR_ALLOC, "domain_create: out of host memory");
  std::memcpy(d->gdims, global_dims, sizeof d->gdims);
  d->nranks = nranks;
  d->rank = rank;
  d->Rz = Rz;
  d->Rt = Rt;
  d->rz = rank % Rz;
  d->rt = rank / Rz;
  d->nl = nlinks;
  d->h = h;
  d->T = T;
  d->Z = Z;
  d->hz = zghost ? h : 0;
  const int edims[4] = {global_dims[0], global_dims[1], Z + 2 * d->hz, T + 2 * h};
  const int ldims[4] = {global_dims[0], global_dims[1], Z, T};
  qexstag_layout *le = nullptr, *ll = nullptr;
  if ((rc = qexstag_layout_create(edims, &le)) || (rc = qexstag_layout_create(ldims, &ll))) {
    if (le) qexstag_layout_destroy(le);
    delete d;
    return rc;
  }
  // the slab's long links carry the global antiperiodic boundary: the
  // 12-real check and the sloppy kernels' long-link signs use global time
  le->g.t0 = d->rt * T - h;
  le->g.L3g = global_dims[3];
  d->ext = le;
  d->local.push_back(ll->g);
  qexstag_layout_destroy(ll);
  void *z = nullptr;
  const size_t lb = sizeof(double2) * 9 * (size_t)le->g.V * nlinks;
  if (cudaMalloc(&z, lb) != cudaSuccess || cudaMalloc((void **)&d->dsum, kDevScalarBytes) != cudaSuccess ||
      cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (z) cudaFree(z);
    if (d->dsum) cudaFree(d->dsum);
    if (d->side) cudaStreamDestroy(d->side);
    if (d->fork) cudaEventDestroy(d->fork);
    qexstag_layout_destroy(le);
    delete d;
    return fail(QEXSTAG_ERR_ALLOC, "domain_create: device allocation failed");
  }
  // unit links to start with (replaced by qexstag_domain_links)
  unit_links_kernel<<<grid_for((long)le->g.V * nlinks), kBlock, 0, stream()>>>((size_t)le->g.V * nlinks,
                                                                               (double2 *)z);
  unit_diag_kernel<<<grid_for(le->g.V), kBlock, 0, stream()>>>(nlinks, le->g.V, (double2 *)z);
  note_launch(2);
  rc = qexstag_links_create(le, nlinks, (const double *)z, QEXSTAG_MEM_DEVICE, 1.0, &d->g);
  cudaFree(z);
  if (rc) {
    cudaFree(d->dsum);
    cudaStreamDestroy(d->side);
    cudaEventDestroy(d->fork);
    cudaEventDestroy(d->join);
    qexstag_layout_destroy(le);
    delete d;
    return rc;
  }
  *out = d;
  return QEXSTAG_OK;
}

int qexstag_domain_create(const int global_dims[4], int nranks, int rank, int nlinks, qexstag_domain **out) {
  return domain_create(global_dims, 1, nranks, rank, nlinks, false, out);
}

int qexstag_domain_create_zt(const int global_dims[4], const int grid[2], int rank, int nlinks,
                             qexstag_domain **out) {
  if (!grid) return fail(QEXSTAG_ERR_ARG, "domain_create_zt: null grid");
  return domain_create(global_dims, grid[0], grid[1], rank, nlinks, true, out);
}

int qexstag_domain_destroy(qexstag_domain *d) {
  if (!d) return QEXSTAG_OK;
  if (d->comm && nccl().ok) nccl().commDestroy(d->comm);
  if (d->hbuf) {
    cudaStreamSynchronize(stream());
    if (d->side) cudaStreamSynchronize(d->side);
    cudaFreeHost(d->hbuf);
  }
  if (d->g) qexstag_links_destroy(d->g);
  if (d->ext) qexstag_layout_destroy(d->ext);
  if (d->dsum) cudaFree(d->dsum);
  if (d->side) {
    cudaStreamSynchronize(d->side);
    cudaStreamDestroy(d->side);
  }
  if (d->fork) cudaEventDestroy(d->fork);
  if (d->join) cudaEventDestroy(d->join);
  delete d;
  return QEXSTAG_OK;
}

int qexstag_domain_local_dims(const qexstag_domain *d, int dims[4]) {
  if (!d || !dims) return fail(QEXSTAG_ERR_ARG, "domain_local_dims: null argument");
  dims[0] = d->gdims[0];
  dims[1] = d->gdims[1];
  dims[2] = d->Z;
  dims[3] = d->T;
  return QEXSTAG_OK;
}

int qexstag_domain_connect_local(qexstag_domain *const *doms, int n) {
  if (!doms || n < 1) return fail(QEXSTAG_ERR_ARG, "domain_connect_local: empty set");
  for (int k = 0; k < n; k++) {
    if (!doms[k] || doms[k]->nranks != n || doms[k]->rank != k)
      return fail(QEXSTAG_ERR_ARG, "domain_connect_local: pass every rank's domain, in rank order");
    if (doms[k]->nl != doms[0]->nl || std::memcmp(doms[k]->gdims, doms[0]->gdims, sizeof doms[0]->gdims) ||
        doms[k]->Rz != doms[0]->Rz || doms[k]->hz != doms[0]->hz)
      return fail(QEXSTAG_ERR_ARG, "domain_connect_local: domains of different lattices");
  }
  for (int k = 0; k < n; k++) {
    qexstag_domain_s *d = doms[k];
    d->up = doms[rank_of(d, d->rz, d->rt + 1)];
    d->down = doms[rank_of(d, d->rz, d->rt - 1)];
    d->zup = doms[rank_of(d, d->rz + 1, d->rt)];
    d->zdown = doms[rank_of(d, d->rz - 1, d->rt)];
    d->connected = true;
  }
  return QEXSTAG_OK;
}

int qexstag_nccl_unique_id(void *id) {
  if (!id) return fail(QEXSTAG_ERR_ARG, "nccl_unique_id: null argument");
  if (!nccl().ok) return fail(QEXSTAG_ERR_STATE, "nccl_unique_id: libnccl.so.2 not available");
  QS_NCCL(nccl().getUniqueId((ncclUniqueId *)id));
  return QEXSTAG_OK;
}

int qexstag_domain_connect_nccl(qexstag_domain *d, const void *id) {
  if (!d || !id) return fail(QEXSTAG_ERR_ARG, "domain_connect_nccl: null argument");
  if (!nccl().ok) return fail(QEXSTAG_ERR_STATE, "domain_connect_nccl: libnccl.so.2 not available");
  if (d->connected) return fail(QEXSTAG_ERR_STATE, "domain_connect_nccl: the domain is already connected");
  ncclUniqueId u;
  std::memcpy(&u, id, sizeof u);
  QS_NCCL(nccl().commInitRank(&d->comm, d->nranks, u, d->rank));
  d->connected = true;
  return QEXSTAG_OK;
}

int qexstag_domain_connect_host(qexstag_domain *d, const qexstag_host_comm *comm) {
  if (!d || !comm || !comm->push_send || !comm->push_recv || !comm->wait_all || !comm->all_reduce_sum)
    return fail(QEXSTAG_ERR_ARG, "domain_connect_host: null domain, communicator or callback");
  if (d->connected) return fail(QEXSTAG_ERR_STATE, "domain_connect_host: the domain is already connected");
  d->hc = *comm;
  d->hostc = true;
  d->connected = true;
  return QEXSTAG_OK;
}

int qexstag_domain_links(qexstag_domain *const *doms, int n, const double *const *links, int mem) {
  int rc;
  if ((rc = check_set(doms, n))) return rc;
  if (!links || (mem != QEXSTAG_MEM_HOST && mem != QEXSTAG_MEM_DEVICE))
    return fail(QEXSTAG_ERR_ARG, "domain_links: bad arguments");
  std::vector<double2 *> base(n);
  for (int k = 0; k < n; k++) {
    qexstag_domain_s *d = doms[k];
    if (!links[k]) return fail(QEXSTAG_ERR_ARG, "domain_links: null links");
    const size_t Vl = (size_t)d->local[0].V, Ve = (size_t)d->ext->g.V;
    const double2 *src = (const double2 *)links[k];
    void *soa = nullptr;
    if (mem == QEXSTAG_MEM_HOST) {
      void *aos;
      if ((rc = d->g->ws.get(kSlotAos, sizeof(double2) * 9 * Vl, &aos)) ||
          (rc = d->g->ws.get(kDmLinks, sizeof(double2) * 9 * Vl * d->nl, &soa)))
        return rc;
      for (int l = 0; l < d->nl; l++) {
        QS_CUDA(cudaMemcpyAsync(aos, links[k] + (size_t)l * 18 * Vl, sizeof(double2) * 9 * Vl,
                                cudaMemcpyHostToDevice, stream()));
        if ((rc = aos_to_soa((const double *)aos, (double2 *)soa + (size_t)l * 9 * Vl, (int)Vl, (int)Vl, 9)))
          return rc;
      }
      src = (const double2 *)soa;
    }
    for (int l = 0; l < d->nl; l++)
      if ((rc = convert(d, src + (size_t)l * 9 * Vl, Vl, d->g->u64 + (size_t)l * 9 * Ve, Ve, 9, true))) return rc;
    base[k] = d->g->u64;
  }
  // ghosts of every link component, both parities
  const int ncomp = 9 * doms[0]->nl;
  for (int par = 0; par < 2; par++)
    if ((rc = exchange(doms, n, base.data(), ncomp, par, stream()))) return rc;
  // the reduced-precision copies the mixed-precision solve iterates with
  for (int k = 0; k < n; k++) {
    free_low_links(doms[k]->g->low);
    if ((rc = build_low_links(doms[k]->g))) return rc;
  }
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

int qexstag_domain_recon12(const qexstag_domain *d) { return (d && d->g && d->g->low.recon12) ? 1 : 0; }

int qexstag_domain_stagD2ee(qexstag_domain *const *doms, int n, double *const *r, const double *const *x, double m2,
                            int mem) {
  int rc;
  if ((rc = check_set(doms, n))) return rc;
  if (!r || !x) return fail(QEXSTAG_ERR_ARG, "domain_stagD2ee: null fields");
  std::vector<double2 *> xe(n), re(n), te(n);
  for (int k = 0; k < n; k++) {
    if ((rc = vec_in(doms[k], kDmIn, x[k], mem, &xe[k])) || (rc = vec_slot_get(doms[k], kDmOut, &re[k])) ||
        (rc = vec_slot_get(doms[k], kDmT, &te[k])))
      return rc;
  }
  if ((rc = schur_set(doms, n, re.data(), xe.data(), te.data(), m2))) return rc;
  for (int k = 0; k < n; k++) {
    // only the even sites of r are written, as stagD2ee does
    const Geom &loc = doms[k]->local[0];
    const size_t Ve = (size_t)doms[k]->ext->g.V;
    if (mem == QEXSTAG_MEM_DEVICE) {
      double2 *full;
      if ((rc = vec_slot_get(doms[k], kDmFull, &full)) || (rc = convert(doms[k], re[k], Ve, full, loc.V, 3, false)))
        return rc;
      for (int c = 0; c < 3; c++)
        QS_CUDA(cudaMemcpyAsync((double2 *)r[k] + (size_t)c * loc.V, full + (size_t)c * loc.V,
                                sizeof(double2) * loc.nh, cudaMemcpyDeviceToDevice, stream()));
    } else {
      double *rh = r[k];
      std::vector<double> keep((size_t)6 * (loc.V - loc.nh));
      std::memcpy(keep.data(), rh + (size_t)6 * loc.nh, keep.size() * sizeof(double));
      if ((rc = vec_out(doms[k], re[k], rh, mem))) return rc;
      std::memcpy(rh + (size_t)6 * loc.nh, keep.data(), keep.size() * sizeof(double));
    }
  }
  QS_CUDA(cudaStreamSynchronize(stream()));
  return QEXSTAG_OK;
}

// CG for stagD2ee(m^2) y = b_e across the domains (cg.nim:55-272, cpNone),
// FP64 from a zero start; x receives y on even sites and zeros on odd sites.
int qexstag_domain_solveEE(qexstag_domain *const *doms, int n, double *const *x, const double *const *b, double m,
                           const qexstag_solver_params *p, qexstag_solver_stats *st_out, int mem) {
  int rc;
  if ((rc = check_set(doms, n))) return rc;
  if (!x || !b || !p) return fail(QEXSTAG_ERR_ARG, "domain_solveEE: null argument");
  const double m2 = m * m;
  std::vector<double2 *> bv(n), xv(n), rv(n), pv(n), ap(n), tv(n);
  for (int k = 0; k < n; k++) {
    qexstag_domain_s *d = doms[k];
    if ((rc = vec_in(d, kDmIn, b[k], mem, &bv[k])) || (rc = vec_slot_get(d, kDmX, &xv[k])) ||
        (rc = vec_slot_get(d, kDmR, &rv[k])) || (rc = vec_slot_get(d, kDmP, &pv[k])) ||
        (rc = vec_slot_get(d, kDmAp, &ap[k])) || (rc = vec_slot_get(d, kDmT, &tv[k])))
      return rc;
    const size_t bytes = sizeof(double2) * 3 * (size_t)d->ext->g.V;
    QS_CUDA(cudaMemsetAsync(xv[k], 0, bytes, stream()));
    QS_CUDA(cudaMemsetAsync(pv[k], 0, bytes, stream()));
    QS_CUDA(cudaMemsetAsync(rv[k], 0, bytes, stream()));
    // sites the sweeps do not write (z ghost rows) stay zero
    QS_CUDA(cudaMemsetAsync(ap[k], 0, bytes, stream()));
    QS_CUDA(cudaMemsetAsync(tv[k], 0, bytes, stream()));
    const int ni = interior_n(d);
    if ((rc = vcopy(interior(d, rv[k]), cv(interior(d, bv[k])), ni)) ||
        (rc = vcopy(interior(d, pv[k]), cv(interior(d, bv[k])), ni)))
      return rc;
  }
  if (p->sloppy != QEXSTAG_SLOPPY_NONE) {
    if (p->sloppy != QEXSTAG_SLOPPY_HALF || n != 1 || doms[0]->hz > 0)
      return fail(QEXSTAG_ERR_ARG, "domain_solveEE: a mixed-precision domain solve takes sloppy HALF, one domain "
                                   "per call and a split along t only");
    qexstag_domain_s *d = doms[0];
    if (!d->g->low.ready) return fail(QEXSTAG_ERR_STATE, "domain_solveEE: set the links first");
    qexstag_solver_stats s2;
    std::memset(&s2, 0, sizeof s2);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream());
    const long long l0 = launch_count();
    double r2 = 0, b2 = 0;
    rc = dot_set(doms, 1, bv.data(), bv.data(), &b2);
    if (!rc) rc = solve_mixed_domain(d, bv[0], xv[0], ap[0], tv[0], m, p, &s2, &r2);
    cudaEventRecord(e1, stream());
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = vec_out(d, xv[0], x[0], mem))) return rc;
    QS_CUDA(cudaStreamSynchronize(stream()));
    if (st_out) {
      *st_out = s2;
      st_out->calls = 1;
      st_out->seconds = ms * 1e-3;
      st_out->flops = (double)(d->nl * 4 * 72 + 60) *
                      ((double)d->gdims[0] * d->gdims[1] * d->gdims[2] * d->gdims[3] / 2) * s2.iterations;
      st_out->r2 = b2 > 0 ? r2 / b2 : 0.0;
      st_out->kernel_launches = launch_count() - l0;
    }
    return r2 <= p->r2req * b2 * 1.0000001 ? QEXSTAG_OK : QEXSTAG_NOT_CONVERGED;
  }
  double b2 = 0;
  if ((rc = dot_set(doms, n, bv.data(), bv.data(), &b2))) return rc;
  if (!std::isfinite(b2)) return fail(QEXSTAG_ERR_NAN, "domain_solveEE: source is not finite");
  const double r2stop = p->r2req * b2;
  const int maxits = p->maxits > 0 ? p->maxits : 50000;
  CgState hs;
  std::memset(&hs, 0, sizeof hs);
  hs.b2 = hs.r2 = hs.rz = b2;
  hs.r2req = p->r2req;
  hs.r2stop = r2stop;
  hs.maxits = maxits;
  hs.done = (b2 > r2stop) ? 0 : 1;
  CgState *st = (CgState *)(doms[0]->dsum + kStateOff);
  if ((rc = write_state(st, hs))) return rc;
  int total = 0;
  for (int k = 0; k < n; k++) total += interior_n(doms[k]);
  const int every = check_interval(total);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, stream());
  auto batch = [&]() -> int {
    int rc2 = QEXSTAG_OK;
    for (int i = 0; i < every && !rc2; i++)
      rc2 = cg_iteration(doms, n, xv.data(), rv.data(), pv.data(), ap.data(), tv.data(), m2, st);
    return rc2;
  };
  // the state is read one batch behind (the next batch is queued first);
  // every rank reads the same all-reduced state, so all queue the same
  // batches, and those past convergence return at once
  StateSnapshot snap;
  if (!hs.done) rc = batch();
  while (!rc && !hs.done) {
    if ((rc = snap.start(st, sizeof(CgState))) || (rc = batch()) || (rc = snap.wait(&hs, sizeof(CgState)))) break;
  }
  cudaEventRecord(e1, stream());
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int its = hs.itn;
  if (!rc && hs.nan) rc = fail(QEXSTAG_ERR_NAN, "domain_solveEE: NaN residual");
  if (rc) return rc;
  // true residual
  for (int k = 0; k < n; k++) {
    // odd sites of the solution are zero
    const size_t Ve = (size_t)doms[k]->ext->g.V, nh = (size_t)doms[k]->ext->g.nh;
    for (int c = 0; c < 3; c++) QS_CUDA(cudaMemsetAsync(xv[k] + c * Ve + nh, 0, sizeof(double2) * nh, stream()));
  }
  if ((rc = schur_set(doms, n, ap.data(), xv.data(), tv.data(), m2))) return rc;
  for (int k = 0; k < n; k++) {
    const int ni = interior_n(doms[k]);
    if ((rc = vsub(interior(doms[k], rv[k]), cv(interior(doms[k], bv[k])), cv(interior(doms[k], ap[k])), ni)))
      return rc;
  }
  double rt2 = 0;
  if ((rc = dot_set(doms, n, rv.data(), rv.data(), &rt2))) return rc;
  for (int k = 0; k < n; k++)
    if ((rc = vec_out(doms[k], xv[k], x[k], mem))) return rc;
  QS_CUDA(cudaStreamSynchronize(stream()));
  if (st_out) {
    std::memset(st_out, 0, sizeof(*st_out));
    st_out->calls = 1;
    st_out->iterations = its;
    st_out->outer_iterations = 1;
    st_out->seconds = ms * 1e-3;
    st_out->flops = (double)(doms[0]->nl * 4 * 72 + 60) * ((double)doms[0]->gdims[0] * doms[0]->gdims[1] *
                                                           doms[0]->gdims[2] * doms[0]->gdims[3] / 2) * its;
    st_out->r2 = b2 > 0 ? rt2 / b2 : 0.0;
  }
  return rt2 <= r2stop * 1.0000001 ? QEXSTAG_OK : QEXSTAG_NOT_CONVERGED;
}

}  // extern "C"
