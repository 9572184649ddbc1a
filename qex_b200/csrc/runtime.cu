// runtime.cu -- error reporting, device selection, stream and the reduction
// scratch shared by all kernels that end in a grid-wide sum.
#include <cstdio>
#include <mutex>
#include <string>

#include "internal.cuh"

namespace qs {

void noalloc_forget(int dev);  // noalloc.cu

namespace {
thread_local std::string g_last_error = "no error";
thread_local cudaStream_t g_stream = nullptr;
thread_local long long g_launches = 0;

struct DeviceRuntime {
  bool ready = false;
  int sms = 148;
  double *partials = nullptr;
  unsigned *tickets = nullptr;
  double *results = nullptr;       // device, kNumResults doubles
  double *host_results = nullptr;  // pinned, kNumResults doubles
};
constexpr int kMaxDevices = 64;
DeviceRuntime g_dev[kMaxDevices];
std::mutex g_mutex;

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

int ensure_runtime(int d) {
  if (d < 0 || d >= kMaxDevices) return fail(QEXSTAG_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceRuntime &r = g_dev[d];
  if (r.ready) return QEXSTAG_OK;
  cudaDeviceProp prop;
  QS_CUDA(cudaGetDeviceProperties(&prop, d));
  r.sms = prop.multiProcessorCount;
  QS_CUDA(cudaMalloc(&r.partials, sizeof(double) * kMaxRedBlocks * 8));
  QS_CUDA(cudaMalloc(&r.tickets, sizeof(unsigned) * kNumTickets));
  QS_CUDA(cudaMemset(r.tickets, 0, sizeof(unsigned) * kNumTickets));
  QS_CUDA(cudaMalloc(&r.results, sizeof(double) * kNumResults));
  QS_CUDA(cudaMemset(r.results, 0, sizeof(double) * kNumResults));
  QS_CUDA(cudaHostAlloc(&r.host_results, sizeof(double) * kNumResults, cudaHostAllocDefault));
  QS_CUDA(cudaDeviceSynchronize());
  r.ready = true;
  return QEXSTAG_OK;
}
}  // namespace

void set_error(const std::string &msg) { g_last_error = msg; }
void note_launch(int n) { g_launches += n; }
long long launch_count() { return g_launches; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return QEXSTAG_ERR_CUDA;
}

cudaStream_t stream() { return g_stream; }

int num_sms() { return g_dev[current_device()].sms; }

double *red_partials() {
  int d = current_device();
  ensure_runtime(d);
  return g_dev[d].partials;
}
unsigned *red_tickets() {
  int d = current_device();
  ensure_runtime(d);
  return g_dev[d].tickets;
}

double *red_results() {
  int d = current_device();
  ensure_runtime(d);
  return g_dev[d].results;
}
double *host_results() {
  int d = current_device();
  ensure_runtime(d);
  return g_dev[d].host_results;
}

int runtime_ready() { return ensure_runtime(current_device()); }

}  // namespace qs

extern "C" {

int qexstag_init(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return qs::cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= n) return qs::fail(QEXSTAG_ERR_ARG, "qexstag_init: no such device");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return qs::cuda_fail(e, "cudaSetDevice");
  return qs::ensure_runtime(device);
}

int qexstag_finalize(void) {
  int d = qs::current_device();
  qs::noalloc_forget(d);
  std::lock_guard<std::mutex> lock(qs::g_mutex);
  qs::DeviceRuntime &r = qs::g_dev[d];
  if (!r.ready) return QEXSTAG_OK;
  cudaDeviceSynchronize();
  cudaFree(r.partials);
  cudaFree(r.tickets);
  cudaFree(r.results);
  cudaFreeHost(r.host_results);
  r = qs::DeviceRuntime();
  return QEXSTAG_OK;
}

int qexstag_set_stream(void *s) {
  qs::g_stream = (cudaStream_t)s;
  return QEXSTAG_OK;
}

const char *qexstag_last_error(void) { return qs::g_last_error.c_str(); }

int qexstag_synchronize(void) {
  QS_CUDA(cudaStreamSynchronize(qs::g_stream));
  return QEXSTAG_OK;
}

}  // extern "C"
