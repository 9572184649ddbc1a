// blas.cu -- layout conversion, FP64 vector updates and deterministic FP64
// reductions on colour-vector fields (QEX's field expressions and
// norm2/redot, src/field/fieldET.nim:648-780, restricted to what the solvers
// use).  All kernels are grid-stride loops over sites; a reduction's
// grid size is fixed for a given site count, so its result is bitwise
// reproducible.
#include "lib.cuh"

namespace qs {

// host AoS double[n][ncomp][2] -> device SoA double2[ncomp][stride]
__global__ void aos_to_soa_kernel(const double2 *__restrict__ aos, double2 *__restrict__ soa, int n,
                                  int stride, int ncomp) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int c = 0; c < ncomp; c++) soa[(size_t)c * stride + i] = aos[(size_t)i * ncomp + c];
}
__global__ void soa_to_aos_kernel(const double2 *__restrict__ soa, double2 *__restrict__ aos, int n,
                                  int stride, int ncomp) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int c = 0; c < ncomp; c++) aos[(size_t)i * ncomp + c] = soa[(size_t)c * stride + i];
}

int aos_to_soa(const double *aos, double2 *soa, int n, int stride, int ncomp) {
  aos_to_soa_kernel<<<grid_for(n), kBlock, 0, stream()>>>((const double2 *)aos, soa, n, stride, ncomp);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}
int soa_to_aos(const double2 *soa, double *aos, int n, int stride, int ncomp) {
  soa_to_aos_kernel<<<grid_for(n), kBlock, 0, stream()>>>(soa, (double2 *)aos, n, stride, ncomp);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

// ---------------------------------------------------------------------------
// elementwise updates on [3][stride] fields, n sites
// ---------------------------------------------------------------------------

enum VOp { kCopy, kZero, kScale, kAxpy, kXpay, kAxpby, kSub };

template <int OP>
__global__ void vop_kernel(double2 *__restrict__ y, int ys, const double2 *__restrict__ x, int xs,
                           const double2 *__restrict__ z, int zs, double a, double b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 *py = y + (size_t)c * ys + i;
      double2 r;
      if (OP == kCopy) {
        r = x[(size_t)c * xs + i];
      } else if (OP == kZero) {
        r = make_double2(0.0, 0.0);
      } else if (OP == kScale) {
        double2 v = *py;
        r = make_double2(a * v.x, a * v.y);
      } else if (OP == kAxpy) {
        double2 v = *py, u = x[(size_t)c * xs + i];
        r = make_double2(fma(a, u.x, v.x), fma(a, u.y, v.y));
      } else if (OP == kXpay) {
        double2 v = *py, u = x[(size_t)c * xs + i];
        r = make_double2(fma(a, v.x, u.x), fma(a, v.y, u.y));
      } else if (OP == kAxpby) {
        double2 v = *py, u = x[(size_t)c * xs + i];
        r = make_double2(fma(a, u.x, b * v.x), fma(a, u.y, b * v.y));
      } else {  // kSub: y = x - z
        double2 u = x[(size_t)c * xs + i], w = z[(size_t)c * zs + i];
        r = make_double2(u.x - w.x, u.y - w.y);
      }
      *py = r;
    }
  }
}

template <int OP>
static int vop(VecD y, CVecD x, CVecD z, double a, double b, int n) {
  vop_kernel<OP><<<grid_for(n), kBlock, 0, stream()>>>(y.p, y.stride, x.p, x.stride, z.p, z.stride,
                                                      a, b, n);
  note_launch();
  QS_LAUNCH_CHECK();
  return QEXSTAG_OK;
}

static const CVecD kNone{nullptr, 0};
int vcopy(VecD y, CVecD x, int n) { return vop<kCopy>(y, x, kNone, 0, 0, n); }
int vzero(VecD y, int n) { return vop<kZero>(y, kNone, kNone, 0, 0, n); }
int vscale(VecD y, double s, int n) { return vop<kScale>(y, kNone, kNone, s, 0, n); }
int vaxpy(VecD y, double a, CVecD x, int n) { return vop<kAxpy>(y, x, kNone, a, 0, n); }
int vxpay(VecD y, CVecD x, double a, int n) { return vop<kXpay>(y, x, kNone, a, 0, n); }
int vaxpby(VecD y, double a, CVecD x, double b, int n) { return vop<kAxpby>(y, x, kNone, a, b, n); }
int vsub(VecD y, CVecD a, CVecD b, int n) { return vop<kSub>(y, a, b, 0, 0, n); }

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------

enum RKind { kNorm2, kRedot, kDiffNorm2 };

template <int K>
__global__ void __launch_bounds__(kBlock)
    reduce_kernel(const double2 *__restrict__ x, int xs, const double2 *__restrict__ y, int ys, int n,
                  double *partials, unsigned *ticket, double *result) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double2 u = x[(size_t)c * xs + i];
      if (K == kNorm2) {
        s = fma(u.x, u.x, s);
        s = fma(u.y, u.y, s);
      } else if (K == kRedot) {
        double2 v = y[(size_t)c * ys + i];
        s = fma(u.x, v.x, s);
        s = fma(u.y, v.y, s);
      } else {
        double2 v = y[(size_t)c * ys + i];
        double dx = u.x - v.x, dy = u.y - v.y;
        s = fma(dx, dx, s);
        s = fma(dy, dy, s);
      }
    }
  }
  double v[1] = {s}, o[1];
  if (grid_reduce<1>(v, partials, ticket, o) && threadIdx.x == 0) *result = o[0];
}

template <int K>
static int reduce(CVecD x, CVecD y, int n, double *host) {
  double *res = red_results();
  int grid = grid_for(n, kBlock, 4);
  reduce_kernel<K><<<grid, kBlock, 0, stream()>>>(x.p, x.stride, y.p, y.stride, n, red_partials(),
                                                 red_tickets(), res);
  note_launch();
  QS_LAUNCH_CHECK();
  if (host) {
    double *h = host_results();
    QS_CUDA(cudaMemcpyAsync(h, res, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    QS_CUDA(cudaStreamSynchronize(stream()));
    *host = h[0];
  }
  return QEXSTAG_OK;
}

int vnorm2(CVecD x, int n, double *host) { return reduce<kNorm2>(x, kNone, n, host); }
int vredot(CVecD x, CVecD y, int n, double *host) { return reduce<kRedot>(x, y, n, host); }
int vdiffnorm2(CVecD a, CVecD b, int n, double *host) { return reduce<kDiffNorm2>(a, b, n, host); }

}  // namespace qs
