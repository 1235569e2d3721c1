// kernels.h -- launch descriptors and launcher entry points of the device
// kernels (internal to libtrtt_b200; the public C ABI is include/trtt_b200.h).
#pragma once

#include <cuda_runtime.h>

#include "trtt_types.h"

namespace trtt {

// Device error bits written by kernels into a flag word.
enum : int {
  TRTT_ERR_SOURCE_PLANE = 1,  // a voxel lies in the source plane (wk == 0)
  TRTT_ERR_BAD_INDEX = 2,     // sparse index out of range
  TRTT_ERR_STALL = 4,         // a bounded wait gave up (tensor-core band kernel)
};

// One (view, weight) contribution to a gate in the transpose.
struct GateEntry {
  int view;
  float w;
};

// The transpose's gate weights of one view: w0 into gate g0, w1 into g1
// (g1 < 0: none).  The same pairs as the per-gate entry lists, by view.
struct GatePair {
  int g0, g1;
  float w0, w1;
};

struct Fwd3DLaunch {
  Params3D P;
  const View3D *views;   // device, nviews entries
  int nviews;
  const float *vol;      // column layout [gate][j][i][k]
  long gate_stride;      // nx*ny*nz
  float *sino;           // [view][nv][nu], accumulated
  long sino_view_stride; // nv*nu
  int band_rows;         // > 0: band kernel (factorised views); 0: per-voxel
  int warps;             // warps per CTA of the band kernel
  int pull = 0;          // closed-form model, nu <= 512: atomic-free band kernel
  int cols = 1;          // closed-form model: 2 = column-pair band kernel
  int tc = 0;            // closed-form model: 1 = tensor-core band kernel (rows chosen by it)
  int *err;              // device error flags
};

struct Back3DLaunch {
  Params3D P;
  const View3D *views;
  const int *gate_ptr;   // ngates+1 offsets into entries
  const GateEntry *entries;
  int ngates;
  int view_lo, view_hi;  // entries outside [view_lo, view_hi) are skipped
  const float *sino;     // detector images of views view_lo..view_hi-1
  long sino_view_stride;
  float *vol;            // column layout, accumulated
  long gate_stride;
  int factorized;        // 1: column kernel; 0: per-voxel kernel
  const GatePair *pairs = nullptr;  // by view index; non-null: all gates in one pass over the views
  int *err;
};

// Direct projector over groups of views related by turns of the volume grid
// (proj3d_group.cu; closed-form model, column-factorised views, one gate).
// `groups` holds 4 view indices per group (members m >= G unused); member m
// sees at view groups[4g]'s footprint of column c the voxel column
// R^{-t_m}(c) (t_m = m for G = 4, 2m for G = 2).
struct GroupFwdLaunch {
  Params3D P;
  const View3D *views;   // device, all views of the plan
  const int *groups;     // device, 4 * ngroups view indices
  int ngroups;
  const float *vol;      // column layout [j][i][k]
  float *sino;           // [view][nv][nu], accumulated
  long sino_view_stride;
  int band_rows;         // R detector rows per CTA
  int usplit, utile;     // u tiles per band and cells per tile (utile <= 256)
  int warps;
  int interleave = 0;    // 1: member profiles interleaved per cell, plain updates where they apply
  int minb = 1;          // groups of 4: 1 CTA per SM (up to 22 warps) or 2 (64 registers per thread)
  int *err;
};

// Transpose over orbits of columns under the group's turns, for the groups
// [g_lo, g_hi) of `groups`.
struct GroupBackLaunch {
  Params3D P;
  const View3D *views;
  const int *groups;
  int g_lo, g_hi;
  int norbits;           // group_orbits(G, nx, ny)
  const float *sino;     // [view][nv][nu], all views of the plan
  long sino_view_stride;
  float *vol;            // column layout, accumulated
  int vec4 = 0;          // 1: nu % 4 == 0 and sino 16-byte aligned (vector loads)
  int *err;
};

// Weighted least-squares data term of a scan in one persistent cooperative
// launch (persist4d.cu; closed-form model, column-factorised views, gates):
// resid = W (H x - y), *cost = 1/2 sum W (H x - y)^2, grad += H^T resid.
struct WlsLaunch {
  Params3D P;
  const View3D *views;
  int nviews;
  const int *gate_ptr;       // ngates+1 offsets into entries
  const GateEntry *entries;
  int ngates;
  const float *vol;          // column layout, gates stacked
  long gate_stride;
  const float *y, *w;        // [view][nv][nu]; w may be null (unit weights)
  float *resid;              // [view][nv][nu] scratch
  float *grad;               // column layout, gates stacked, accumulated
  double *cost_parts;        // one per band item
  double *cost;              // device, written
  unsigned *queue;           // [0] next item, [1] finished band items; zero before launch
  int band_rows;
  int ctas_per_sm;           // 1 or 2 (0: 1): register budget of 128 or 64 per thread
  int extra_wait;            // column items also wait for this many band items (test hook)
  long long wait_ns;         // bound of that wait
  int *err;
  const GatePair *pairs;      // by view; non-null with several gates: column items over all gates
  // filled by launch_wls_persistent
  int nbands, kchunks, n_band_items, n_col_items, lock_spread, gates_mode;
};
size_t wls_smem(int nu, int band_rows);
size_t wls_gates_smem(int nu, int ngates, int kp, int gates_mode);
size_t band_fast_smem(int nu, int band_rows, int warps);
// Floats of shared memory per warp of the all-gates transpose: the profile
// row (nu, rounded up to 4) and the per-gate sums and compensations.
__host__ __device__ inline size_t back_gates_row(int nu, int ngates, int kp)
{
  return (size_t)((nu + 3) & ~3) + 2 * (size_t)ngates * 64 * kp;
}
// Spread mode of the band item: row locks for voxel columns of 128 voxels
// or more, shared atomics below (measured: 256^3 -> 512^2 83 -> 74 ms per
// 360 views with locks; 128x128x64 -> 256^2 8.4 -> 9.9 ms, so atomics there).
inline bool band_lock_spread(const Params3D &P) { return P.nz >= 128; }
int wls_kp(int nz);
cudaError_t launch_wls_persistent(WlsLaunch L, int sms, cudaStream_t st);

size_t group_fwd_smem(int G, int band_rows, int utile, int warps);
int group_fwd_warps(int G, int band_rows, int utile, int minb);
int group_orbits(int G, int nx, int ny);
cudaError_t launch_fwd3d_group(const GroupFwdLaunch &L, int G, cudaStream_t st);
cudaError_t launch_back3d_group(const GroupBackLaunch &L, int G, cudaStream_t st);

cudaError_t launch_fwd3d(const Fwd3DLaunch &L, cudaStream_t st);
cudaError_t launch_back3d(const Back3DLaunch &L, cudaStream_t st);
// source-plane test of every column of column-factorised views (err |= flag)
cudaError_t launch_check_columns(const Params3D &P, const View3D *views, int nviews, int *err,
                                 cudaStream_t st);
// closed-form model on factorised views, packed FP32x2 (proj3d_fast.cu)
cudaError_t launch_fwd3d_fast(const Fwd3DLaunch &L, cudaStream_t st);
cudaError_t launch_back3d_fast(const Back3DLaunch &L, cudaStream_t st);

// Layout / precision conversions (convert.cu).
// XYZ layout is the reference's [k][j][i] (x fastest); column layout is
// [j][i][k] (k fastest).  `nb` volumes are converted back to back.
cudaError_t xyz_f64_to_col_f32(const double *src, float *dst, int nx, int ny,
                               int nz, int nb, cudaStream_t st);
cudaError_t xyz_f32_to_col_f32(const float *src, float *dst, int nx, int ny,
                               int nz, int nb, cudaStream_t st);
cudaError_t col_f32_add_to_xyz_f64(const float *src, double *dst, int nx,
                                   int ny, int nz, int nb, cudaStream_t st);
cudaError_t col_f32_add_to_xyz_f32(const float *src, float *dst, int nx,
                                   int ny, int nz, int nb, cudaStream_t st);
cudaError_t f64_to_f32(const double *src, float *dst, long n, cudaStream_t st);
cudaError_t f32_add_to_f64(const float *src, double *dst, long n, cudaStream_t st);

// Tensor-core band kernel of the direct projector (closed-form model,
// column-factorised views): its detector-row band height for an nu x nv
// detector, 0 if the detector is too wide for it (nu > 2048).
int fwd3d_tc_band_rows(int nu, int nv);
cudaError_t launch_fwd3d_tc(const Fwd3DLaunch &L, cudaStream_t st);

}  // namespace trtt
