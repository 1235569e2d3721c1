// noalloc.cu -- allocation-free variant of the cone-beam direct projector.
//
// Some callers cannot call cudaMalloc: real-time or embedded hosts that
// forbid device allocation after start-up (cudaMalloc can synchronise the
// whole device and stall the streams of other work), and frameworks whose
// device memory belongs to their own pool allocator, which must not see a
// library allocate behind its back.  The plan API allocates its per-view
// geometry table on the device; this entry point instead keeps that table
// (and its error word) in one file-scope device array, so the call
// allocates nothing.  The caller still passes the input volume and the
// output detector stack.
//
// Limits and sharing:
//  * at most TRTT_B200_NOALLOC_MAX_VIEWS (2048) views per call, i.e. 2048
//    geometry records of 336 bytes plus one error word: 688,384 bytes of
//    device memory, held by every GPU that loads the library until exit;
//  * every call reuses the same array (it keeps the last call's contents;
//    the error word is cleared by each call), so calls that overlap on the
//    GPU -- on two streams, or from two host threads -- race on it.  Host
//    threads are serialised by a mutex and the call returns only after the
//    projection has completed (it reads the error word back and waits for
//    the stream);
//  * the first call on each device looks the array's device address up
//    (cudaGetSymbolAddress, which may load the module); make that first call
//    before any stream capture begins.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "host3d.h"
#include "kernels.h"
#include "runtime.h"
#include "trtt_b200.h"

using namespace trtt;

namespace {

constexpr long kMaxViews = TRTT_B200_NOALLOC_MAX_VIEWS;
constexpr size_t kErrOffset = 0;     // error word
constexpr size_t kViewsOffset = 256; // geometry records (256-byte aligned)
constexpr size_t kScratchBytes = kViewsOffset + sizeof(View3D) * kMaxViews;

// The scratch array: error word at offset 0, View3D records at offset 256.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};   // device address per device
View3D g_host_views[kMaxViews];           // host staging (no heap allocation)

}  // namespace

extern "C" int trtt_b200_cb3d_cubic_forward_noalloc(const float *vol_columns, float *sino,
                                                    long nx, long ny, long nz, double s_scl,
                                                    int s_deg, long nu, long nv, double u_scl,
                                                    double v_scl, long nviews, const double *xos,
                                                    const double *xsd, void *stream)
{
  clear_error();
  if (!vol_columns || !sino || !xos || !xsd) return fail("cb3d_cubic_forward_noalloc: null argument");
  if (nviews > kMaxViews)
    return fail("cb3d_cubic_forward_noalloc: at most " + std::to_string(kMaxViews) +
                " views per call (the scratch array is static); got " + std::to_string(nviews));
  if (const char *why = check_sizes3d(nx, ny, nz, nu, nv, nviews))
    return fail(std::string("cb3d_cubic_forward_noalloc: ") + why);
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  TRTT_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail("cb3d_cubic_forward_noalloc: device index out of range");
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    TRTT_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = p;
  }
  unsigned char *base = static_cast<unsigned char *>(g_scratch_addr[dev]);
  int *err_dev = reinterpret_cast<int *>(base + kErrOffset);
  View3D *views_dev = reinterpret_cast<View3D *>(base + kViewsOffset);
  cudaStream_t st = (cudaStream_t)stream;

  Params3D P = make_params(GEOM_CONE, nx, ny, nz, s_scl, s_deg, nullptr, 0, 1.0, 0.0, nu, nv,
                           u_scl, v_scl);
  bool fact = true;
  for (long v = 0; v < nviews; ++v) {
    make_view3d(P, xos + 12 * v, xsd + 12 * v, g_host_views[v]);
    fact = fact && g_host_views[v].factorized;
  }
  TRTT_CK(cudaMemcpyAsync(views_dev, g_host_views, sizeof(View3D) * nviews,
                          cudaMemcpyHostToDevice, st));
  TRTT_CK(cudaMemsetAsync(err_dev, 0, sizeof(int), st));
  Fwd3DLaunch L;
  L.P = P;
  L.views = views_dev;
  L.nviews = (int)nviews;
  L.vol = vol_columns;
  L.gate_stride = nx * ny * nz;
  L.sino = sino;
  L.sino_view_stride = nu * nv;
  int rows = 0, warps = 16;
  choose_band((int)nu, (int)nv, rows, warps);
  L.band_rows = fact ? rows : 0;
  L.warps = warps;
  L.err = err_dev;
  TRTT_CK(launch_fwd3d(L, st));
  count_launch();
  int herr = 0;
  TRTT_CK(cudaMemcpyAsync(&herr, err_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  if (herr & TRTT_ERR_SOURCE_PLANE)
    return fail("cb3d_cubic_forward_noalloc: a voxel lies in the source plane (wk == 0)");
  if (herr) return fail("cb3d_cubic_forward_noalloc: device error flag set");
  return 0;
}
