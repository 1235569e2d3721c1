// runtime.cu -- device context, scratch buffers and error reporting of
// libtrtt_b200.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>

#include "runtime.h"

namespace trtt {

std::atomic<long> g_launches{0};

static thread_local std::string t_last_error;

void set_error(const std::string &msg) { t_last_error = msg; }
void clear_error() { t_last_error.clear(); }

int fail(const std::string &msg)
{
  set_error(msg);
  return -1;
}

int fail_cuda(cudaError_t e, const char *what)
{
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return fail(m);
}

bool dim_ok(long n) { return n > 0 && n < (1L << 30); }

cudaError_t DevBuf::ensure(size_t need)
{
  if (need <= bytes && p != nullptr) return cudaSuccess;
  if (p) {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  size_t want = need < 256 ? 256 : need;
  cudaError_t e = cudaMalloc(&p, want);
  if (e == cudaSuccess) bytes = want;
  return e;
}

void DevBuf::release()
{
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

cudaError_t DropIn::init()
{
  if (ready) return cudaSuccess;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaErrorNoDevice;
  const char *env = std::getenv("TRTT_B200_DEVICE");
  if (env) {
    device = std::atoi(env);
  } else {
    e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
  }
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  // The copy stream also runs the small FP32 <-> FP64 conversion kernels
  // between its copies.  The projector kernels occupy every SM (one CTA of
  // up to 219 KB of shared memory per SM), so at default priority a
  // conversion waited for a whole kernel to drain and the copies fell behind
  // (11 ms of trailing copies after a 360-view direct projection); at the
  // greatest priority it takes the next SM that frees up.
  int prio_least = 0, prio_greatest = 0;
  e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (e != cudaSuccess) return e;
  e = cudaStreamCreateWithPriority(&copy, cudaStreamNonBlocking, prio_greatest);
  if (e != cudaSuccess) return e;
  e = cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  for (int i = 0; i < kEvents; ++i) {
    e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  ready = true;
  return cudaSuccess;
}

DropIn &dropin()
{
  static DropIn *d = new DropIn();  // never destroyed: outlives static teardown
  return *d;
}

}  // namespace trtt

extern "C" {

const char *trtt_b200_last_error(void) { return trtt::t_last_error.c_str(); }

const char *trtt_b200_version(void) { return "trtt_b200 0.1 (sm_100a)"; }

long trtt_b200_launch_count(void) { return trtt::g_launches.load(); }

}  // extern "C"
