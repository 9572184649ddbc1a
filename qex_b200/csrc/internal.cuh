// internal.cuh -- shared types and device helpers of the sm_100a staggered
// library.  Device data layout (structure of arrays, site index = QEX's V=1
// checkerboard index, even sites first):
//   colour vector, FP64: double2 [3][stride]  (colour-major; a full field has
//                         stride V, an even- or odd-only block stride V/2)
//   links, FP64:         double2 [nlinks][9][V]  (element e = 3*row+col)
// Reduced-precision link and vector formats are declared in mixed.cuh.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <string>

#include "../../include/qexstag.h"

namespace qs {

constexpr int kBlock = 256;  // threads per block of the streaming kernels

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------

struct Geom {
  int L[4];
  int stride[4];  // lexicographic strides: 1, L0, L0*L1, L0*L1*L2
  int V;
  int nh;  // sites per parity (V/2; all L are even)
  // n / L[d] = umulhi(n, mag[d]) >> shf[d] for 0 <= n < 2^31 (d = 0, 1, 2):
  // shf = floor(log2 L) and mag = ceil(2^(32+shf) / L), or mag = 2^31 and
  // shf = log2(L) - 1 when L is a power of two (set by set_fastdiv)
  unsigned mag[3];
  int shf[3];
  // time slice x3 of this lattice is slice (x3 + t0) mod L3g of the lattice
  // whose antiperiodic boundary the folded phases carry: 0 and L[3] for a
  // whole lattice; a domain's extended slab sets its own offset
  int t0, L3g;
};

inline void set_fastdiv(Geom &g) {
  for (int d = 0; d < 3; d++) {
    const unsigned L = (unsigned)g.L[d];
    int s = 0;
    while ((2u << s) <= L) s++;  // floor(log2 L)
    if ((L & (L - 1)) == 0) {
      g.mag[d] = 1u << 31;
      g.shf[d] = s - 1;
    } else {
      g.mag[d] = (unsigned)((((unsigned long long)1 << (32 + s)) + L - 1) / L);
      g.shf[d] = s;
    }
  }
}

__device__ __forceinline__ int fdiv(const Geom &g, int d, int n) {
  return (int)(__umulhi((unsigned)n, g.mag[d]) >> g.shf[d]);
}

// Coordinates and lex index of the k-th site of parity par.  Follows
// qlayout.nim:108-136 with innerGeom = 1: idx = (lex + par*V)/2, so the
// parity-par site k has lex 2k or 2k+1, whichever has parity par (L0 even).
__device__ __forceinline__ void site_coords(const Geom &g, int par, int k, int x[4], int &lex) {
  int l0 = 2 * k;
  int t = fdiv(g, 0, l0);
  int x0 = l0 - t * g.L[0];
  int t2 = fdiv(g, 1, t);
  x[1] = t - t2 * g.L[1];
  int t3 = fdiv(g, 2, t2);
  x[2] = t2 - t3 * g.L[2];
  x[3] = t3;
  int p0 = (x[1] + x[2] + x[3]) & 1;  // parity of lex l0 (x0 even)
  int bump = p0 ^ par;
  x[0] = x0 + bump;
  lex = l0 + bump;
}

// Half-index (within the opposite parity) of x + d*mu, periodic; |d| <= 3 < L.
__device__ __forceinline__ int nbr_half(const Geom &g, const int x[4], int lex, int mu, int d) {
  int xm = x[mu];
  int xn = xm + d;
  if (xn >= g.L[mu]) xn -= g.L[mu];
  if (xn < 0) xn += g.L[mu];
  return (lex + (xn - xm) * g.stride[mu]) >> 1;
}

template <int NL>
struct Hop {
  static __device__ __forceinline__ int mu(int l) { return NL == 8 ? (l >> 1) : l; }
  static __device__ __forceinline__ int len(int l) { return NL == 8 ? ((l & 1) ? 3 : 1) : 1; }
};

// ---------------------------------------------------------------------------
// complex helpers (double2 / float2 as (re, im))
// ---------------------------------------------------------------------------

__device__ __forceinline__ double2 cmadd(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc += conj(a) * b
__device__ __forceinline__ double2 cjmadd(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ float2 cmadd(float2 acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ float2 cjmadd(float2 acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(-a.y, b.x, acc.y);
  return acc;
}

// Programmatic dependent launch: block until the kernel before this one in
// the stream has completed and its writes are visible.  Kernels that start
// with it may be launched with launch_pdl, which lets the GPU schedule them
// while the previous kernel drains; under an ordinary launch it returns at
// once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// read-only, streaming loads
__device__ __forceinline__ double2 ldg(const double2 *p) { return __ldg(p); }
__device__ __forceinline__ float2 ldg(const float2 *p) { return __ldg(p); }
__device__ __forceinline__ float4 ldg(const float4 *p) { return __ldg(p); }
__device__ __forceinline__ uint4 ldg(const uint4 *p) { return __ldg(p); }
__device__ __forceinline__ uint2 ldg(const uint2 *p) { return __ldg(p); }
__device__ __forceinline__ unsigned ldg(const unsigned *p) { return __ldg(p); }
// links are streamed once per sweep: do not keep them in L1
__device__ __forceinline__ double2 ldlink(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ float4 ldlink(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 ldlink(const float2 *p) { return __ldcs(p); }
__device__ __forceinline__ uint4 ldlink(const uint4 *p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ldlink(const uint2 *p) { return __ldcs(p); }
__device__ __forceinline__ unsigned ldlink(const unsigned *p) { return __ldcs(p); }

// ---------------------------------------------------------------------------
// deterministic grid reduction: block partials, last block sums them in a
// fixed order.  partials holds NV*gridDim.x doubles; ticket is zero on entry
// and is reset by the last block.  Returns true (in every thread of the last
// block) with out[] valid in thread 0.
// ---------------------------------------------------------------------------

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh /* NV*32 */) {
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double s = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    v[j] = s;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; j++) sh[j * 32 + w] = v[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int j = 0; j < NV; j++) {
      double s = 0.0;
      for (int i = 0; i < nw; i++) s += sh[j * 32 + i];
      v[j] = s;
    }
  }
}

template <int NV>
__device__ bool grid_reduce(double (&v)[NV], double *partials, unsigned *ticket,
                            double (&out)[NV]) {
  __shared__ double sh[NV * 32];
  __shared__ bool last;
  block_sum<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; j++) partials[j * gridDim.x + blockIdx.x] = v[j];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double w[NV];
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
      s += __ldcg(partials + j * gridDim.x + i);
    w[j] = s;
  }
  block_sum<NV>(w, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; j++) out[j] = w[j];
    *ticket = 0u;
  }
  return true;
}

// ---------------------------------------------------------------------------
// CG scalars kept on the device so that iterations run without host syncs
// (cg.nim:174-240 with cpNone: z = r, q = p, rz = r2).
// ---------------------------------------------------------------------------

struct CgState {
  double rz;      // r.r at the top of the current iteration
  double beta;    // beta of the next p update
  double alpha;
  double pAp;
  double r2;      // latest |r|^2
  double b2;
  double r2req;   // set by the host
  double r2stop;  // r2req * b2
  double r2max;   // largest |r|^2 since the last reliable update (mixed)
  double r2ref;   // reliable-update reference |r|^2 (mixed)
  int itn;
  int maxits;     // set by the host
  int done;       // 1 once converged, out of iterations or NaN
  int nan;
  int reliable;   // mixed: number of reliable updates done
  int pad[3];
};

// ---------------------------------------------------------------------------
// host side: error reporting and per-device runtime
// ---------------------------------------------------------------------------

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
cudaStream_t stream();
int num_sms();
// Scratch for reductions: partial sums and tickets, reused by every call on
// the library's stream (calls on one stream are ordered).
double *red_partials();   // kMaxRedBlocks * 8 doubles
unsigned *red_tickets();  // kNumTickets unsigned, all zero between kernels
constexpr int kMaxRedBlocks = 4096;
constexpr int kNumTickets = 64;
constexpr int kNumResults = 64;
double *red_results();   // device doubles for reduction results
double *host_results();  // pinned host mirror

#define QS_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::qs::cuda_fail(e_, #call); \
  } while (0)

#define QS_LAUNCH_CHECK() QS_CUDA(cudaGetLastError())

// count of kernels this thread has launched through the library
void note_launch(int n = 1);
long long launch_count();

// launch a kernel that begins with pdl_wait() with programmatic stream
// serialisation on the library's stream
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), int grid, int block, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream();
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, ((KArgs)args)...);
}

inline int grid_for(long n, int block = kBlock, int per_sm = 8) {
  long b = (n + block - 1) / block;
  long cap = (long)num_sms() * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace qs

// handles
struct qexstag_layout_s {
  qs::Geom g;
  int device;
};
