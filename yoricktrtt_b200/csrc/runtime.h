// runtime.h -- host runtime shared by the C ABI translation units: device
// context, cached device buffers, error reporting, launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdio>
#include <mutex>
#include <string>

namespace trtt {

// Thread-local last-error message.
void set_error(const std::string &msg);
void clear_error();

// Count of kernel launches issued by the library.
extern std::atomic<long> g_launches;
inline void count_launch(long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Growable device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need);
  void release();
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Process-wide state of the drop-in (host-buffer) entry points: one device,
// one stream, scratch buffers reused across calls, serialised by a mutex
// (the reference plugin is single-threaded and synchronous).
struct DropIn {
  std::mutex mu;
  bool ready = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;  // host<->device copies that overlap the kernels (greatest priority)
  cudaStream_t stream2 = nullptr;  // second kernel stream: view chunks of the direct projection
  int sms = 148;                 // streaming multiprocessors of `device`
  // ev[0], ev[1]: copy stream start / end; ev[2 + c]: view chunk c (at most
  // kChunks); ev[kEvIn]: the input upload started early on the copy stream;
  // ev[kEvents - 2], ev[kEvents - 1]: second kernel stream start / end
  static constexpr int kChunks = 31;
  static constexpr int kEvIn = kChunks + 2;
  static constexpr int kEvents = kChunks + 5;
  cudaEvent_t ev[kEvents] = {};
  DevBuf in64, out64, vol32, det32, geom, gates, aux, err, grp, xyz32;
  // Pinned staging ring for pageable host arrays (the arrays of a Yorick
  // caller): two slots of kStageBytes, each with the event of its last copy.
  static constexpr size_t kStageBytes = 32u << 20;
  void *stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ev[2] = {};
  cudaError_t init();
  cudaError_t init_stage();
};
DropIn &dropin();

// True when p is ordinary pageable host memory (not allocated or registered
// by CUDA, not device memory): copies from it are staged by the driver at a
// fraction of the DMA speed.
bool host_pageable(const void *p);

// dst (device) <- src (host) on stream s.  From pinned (or device) memory
// one asynchronous copy; from pageable memory of at least 4 MB the bytes pass
// through D's pinned staging ring (host threads fill a slot while the
// previous slot's DMA runs).  Returns when src may be reused; the copies may
// still be in flight on s.
cudaError_t upload_host(DropIn &D, void *dst, const void *src, size_t bytes, cudaStream_t s);

// out[i] += (double)src[i] for i < n (src on the device, out pageable host
// memory): the FP32 values come back through the pinned staging ring and
// host threads add each slot while the next slot's DMA runs.  The same
// FP64 additions as on the device.  Synchronous.
cudaError_t download_add(DropIn &D, double *out, const float *src, long n, cudaStream_t s);

// Report a CUDA error and return -1 (for use in `return fail_cuda(...)`).
int fail_cuda(cudaError_t e, const char *what);
int fail(const std::string &msg);

// Check that a long dimension is positive and fits the kernels' int indices.
bool dim_ok(long n);

}  // namespace trtt

#define TRTT_CK(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return trtt::fail_cuda(e_, #call); \
  } while (0)
