// runtime.cu -- device context, scratch buffers and error reporting of
// libtrtt_b200.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

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

cudaError_t DropIn::init_stage()
{
  for (int i = 0; i < 2; ++i) {
    if (stage[i]) continue;
    cudaError_t e = cudaHostAlloc(&stage[i], kStageBytes, cudaHostAllocPortable);
    if (e != cudaSuccess) return e;
    e = cudaEventCreateWithFlags(&stage_ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

bool host_pageable(const void *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the non-sticky error of an unknown pointer
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

namespace {

// fn(lo, hi) over [0, n) split among up to 16 host threads (one slice each).
template <typename F>
void host_parallel(long n, F fn)
{
  const long min_slice = 1L << 18;
  unsigned hw = std::thread::hardware_concurrency();
  long nt = std::min<long>(hw ? hw : 1, 16);
  nt = std::max<long>(1, std::min<long>(nt, n / min_slice));
  if (nt <= 1) {
    fn(0L, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  const long per = (n + nt - 1) / nt;
  for (long t = 1; t < nt; ++t) {
    const long lo = t * per, hi = std::min(n, lo + per);
    if (lo >= hi) continue;
    try {
      th.emplace_back(fn, lo, hi);
    } catch (...) {
      fn(lo, hi);  // no thread to be had: this slice on the calling thread
    }
  }
  fn(0L, std::min(n, per));
  for (auto &x : th) x.join();
}

}  // namespace

cudaError_t upload_host(DropIn &D, void *dst, const void *src, size_t bytes, cudaStream_t s)
{
  if (bytes < (4u << 20) || !host_pageable(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  cudaError_t e = D.init_stage();
  if (e != cudaSuccess) return e;
  const char *sp = static_cast<const char *>(src);
  char *dp = static_cast<char *>(dst);
  int k = 0;
  for (size_t off = 0; off < bytes; off += DropIn::kStageBytes, ++k) {
    const int slot = k & 1;
    const size_t len = std::min(DropIn::kStageBytes, bytes - off);
    e = cudaEventSynchronize(D.stage_ev[slot]);  // the slot's previous copy has left it
    if (e != cudaSuccess) return e;
    char *stg = static_cast<char *>(D.stage[slot]);
    host_parallel((long)len, [&](long lo, long hi) { std::memcpy(stg + lo, sp + off + lo, (size_t)(hi - lo)); });
    e = cudaMemcpyAsync(dp + off, stg, len, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(D.stage_ev[slot], s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t download_add(DropIn &D, double *out, const float *src, long n, cudaStream_t s)
{
  cudaError_t e = D.init_stage();
  if (e != cudaSuccess) return e;
  const long chunk = (long)(DropIn::kStageBytes / sizeof(float));
  const long nchunks = (n + chunk - 1) / chunk;
  auto issue = [&](long k) -> cudaError_t {
    const int slot = (int)(k & 1);
    const long lo = k * chunk, len = std::min(chunk, n - lo);
    cudaError_t r = cudaEventSynchronize(D.stage_ev[slot]);  // no upload still reads the slot
    if (r != cudaSuccess) return r;
    r = cudaMemcpyAsync(D.stage[slot], src + lo, sizeof(float) * len, cudaMemcpyDeviceToHost, s);
    if (r != cudaSuccess) return r;
    return cudaEventRecord(D.stage_ev[slot], s);
  };
  if (nchunks > 0 && (e = issue(0)) != cudaSuccess) return e;
  for (long k = 0; k < nchunks; ++k) {
    // slot (k+1) & 1 held chunk k-1, whose additions are done
    if (k + 1 < nchunks && (e = issue(k + 1)) != cudaSuccess) return e;
    const int slot = (int)(k & 1);
    e = cudaEventSynchronize(D.stage_ev[slot]);
    if (e != cudaSuccess) return e;
    const float *stg = static_cast<const float *>(D.stage[slot]);
    double *o = out + k * chunk;
    const long len = std::min(chunk, n - k * chunk);
    host_parallel(len, [&](long lo, long hi) {
      for (long i = lo; i < hi; ++i) o[i] += (double)stg[i];
    });
  }
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
