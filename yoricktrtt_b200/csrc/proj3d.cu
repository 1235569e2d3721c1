// proj3d.cu -- sm_100a kernels of the 3D B-spline projector pair for views
// whose transaxial footprint depends on k (general xforms: tilted or
// helical orbits), both footprint models, and the geometry pre-check of
// column-factorised views.
//
// Direct (k_fwd3d_vox): one thread per voxel and view adds its footprint
// into the detector image (FP32 global atomics).  Transpose (k_back3d_vox):
// one thread per voxel gathers over the views of its gate (Kahan sums),
// atomic-free.  Column-factorised views (circular orbits, the reference's
// own scans) take the band and column kernels of proj3d_fast.cu and
// proj3d_group.cu.  Every kernel uses the weights of geom3d.cuh, so each
// pair is an exact adjoint up to FP32 rounding.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "geom3d.cuh"
#include "kernels.h"

namespace trtt {

// Value of voxel k of column `col` for view V (temporal interpolation of the
// 4D path folded into the read: w0 * gate g0 + w1 * gate g1).
__device__ __forceinline__ float voxel_value(const float *__restrict__ vol,
                                             long gate_stride, const View3D &V,
                                             long idx)
{
  float x = __ldg(vol + (long)V.g0 * gate_stride + idx);
  if (V.w1 != 0.0f) {
    float y = __ldg(vol + (long)V.g1 * gate_stride + idx);
    return fmaf(V.w0, x, V.w1 * y);
  }
  return V.w0 == 1.0f ? x : V.w0 * x;
}

// ---------------------------------------------------------------------------
// General xforms (transaxial footprint depends on k): per-voxel kernels.
// The direct projector scatters with FP32 atomics into the view's detector
// image; the transpose gathers per voxel (atomic-free).
// ---------------------------------------------------------------------------
template <int GEOM, int MODEL>
__global__ void __launch_bounds__(256)
k_fwd3d_vox(const Params3D P, const View3D *__restrict__ views,
            const float *__restrict__ vol, long gate_stride,
            float *__restrict__ sino, long sino_view_stride,
            int *__restrict__ err)
{
  const long nvox = (long)P.nx * P.ny * P.nz;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nvox) return;
  const View3D &V = views[blockIdx.y];
  const float x = voxel_value(vol, gate_stride, V, idx);
  if (x == 0.0f) return;
  const int k = (int)(idx % P.nz);
  const int col = (int)(idx / P.nz);
  const int i = col % P.nx, j = col / P.nx;
  ColGeo<MODEL> c;
  column_geo<GEOM, MODEL>(P, V, i, j, k, c);
  if (c.bad) {
    atomicOr(err, TRTT_ERR_SOURCE_PLANE);
    return;
  }
  if (c.vax.n <= 0) return;
  typename AxisOf<MODEL>::type ax;
  float rho0;
  if (!voxel_u<GEOM, MODEL>(P, V, c, k, ax, rho0)) return;
  float *img = sino + (long)blockIdx.y * sino_view_stride;
  const float xr = x * rho0;
  for (int m = 0; m < c.vax.n; ++m) {
    const float wvm = axis_weight<MODEL>(c.vax, m, P) * xr;
    float *row = img + (long)(c.vax.lo + m) * P.nu + ax.lo;
    for (int l = 0; l < ax.n; ++l) atomicAdd(row + l, wvm * axis_weight<MODEL>(ax, l, P));
  }
}

template <int GEOM, int MODEL>
__global__ void __launch_bounds__(256)
k_back3d_vox(const Params3D P, const View3D *__restrict__ views,
             const int *__restrict__ gate_ptr, const GateEntry *__restrict__ entries,
             int view_lo, int view_hi,
             const float *__restrict__ sino, long sino_view_stride,
             float *__restrict__ vol, long gate_stride, int *__restrict__ err)
{
  const long nvox = (long)P.nx * P.ny * P.nz;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nvox) return;
  const int gate = blockIdx.z;
  const int k = (int)(idx % P.nz);
  const int col = (int)(idx / P.nz);
  const int i = col % P.nx, j = col / P.nx;
  Kahan acc;
  for (int e = gate_ptr[gate]; e < gate_ptr[gate + 1]; ++e) {
    const GateEntry ge = entries[e];
    if (ge.view < view_lo || ge.view >= view_hi) continue;
    const View3D &V = views[ge.view];
    ColGeo<MODEL> c;
    column_geo<GEOM, MODEL>(P, V, i, j, k, c);
    if (c.bad) {
      atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      continue;
    }
    if (c.vax.n <= 0) continue;
    typename AxisOf<MODEL>::type ax;
    float rho0;
    if (!voxel_u<GEOM, MODEL>(P, V, c, k, ax, rho0)) continue;
    const float *img = sino + (long)(ge.view - view_lo) * sino_view_stride;
    float s = 0.f;
    for (int m = 0; m < c.vax.n; ++m) {
      const float *row = img + (long)(c.vax.lo + m) * P.nu + ax.lo;
      float t = 0.f;
      for (int l = 0; l < ax.n; ++l) t = fmaf(axis_weight<MODEL>(ax, l, P), __ldg(row + l), t);
      s = fmaf(axis_weight<MODEL>(c.vax, m, P), t, s);
    }
    acc.add(ge.w * rho0 * s);
  }
  vol[(long)gate * gate_stride + idx] += acc.value();
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
template <int GEOM, int MODEL>
static cudaError_t launch_fwd(const Fwd3DLaunch &L, cudaStream_t st)
{
  const long nvox = (long)L.P.nx * L.P.ny * L.P.nz;
  dim3 grid((unsigned)((nvox + 255) / 256), L.nviews);
  k_fwd3d_vox<GEOM, MODEL><<<grid, 256, 0, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino,
                                                L.sino_view_stride, L.err);
  return cudaGetLastError();
}

template <int GEOM, int MODEL>
static cudaError_t launch_back(const Back3DLaunch &L, cudaStream_t st)
{
  const long nvox = (long)L.P.nx * L.P.ny * L.P.nz;
  dim3 grid((unsigned)((nvox + 255) / 256), 1, L.ngates);
  k_back3d_vox<GEOM, MODEL><<<grid, 256, 0, st>>>(L.P, L.views, L.gate_ptr, L.entries, L.view_lo, L.view_hi, L.sino,
                                                 L.sino_view_stride, L.vol, L.gate_stride, L.err);
  return cudaGetLastError();
}

// Geometry pre-check of column-factorised views: the source-plane
// condition of every column of every view, evaluated by the same
// column_geo() the projectors use, so that a caller can learn before any
// projection whether the call will fail.
template <int GEOM, int MODEL>
__global__ void k_check_columns(const Params3D P, const View3D *__restrict__ views, int nviews,
                                int *__restrict__ err)
{
  const long ncols = (long)P.nx * P.ny;
  const long total = ncols * nviews;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int v = (int)(t / ncols);
    const int col = (int)(t - (long)v * ncols);
    ColGeo<MODEL> c;
    column_geo<GEOM, MODEL>(P, views[v], col % P.nx, col / P.nx, 0, c);
    if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
  }
}

cudaError_t launch_check_columns(const Params3D &P, const View3D *views, int nviews, int *err,
                                 cudaStream_t st)
{
  const long total = (long)P.nx * P.ny * nviews;
  long b = (total + 255) / 256;
  if (b > 148L * 16) b = 148L * 16;
  const unsigned grid = (unsigned)(b > 0 ? b : 1);
  if (P.geom == GEOM_CONE) {
    if (P.model == MODEL_TABLE) k_check_columns<GEOM_CONE, MODEL_TABLE><<<grid, 256, 0, st>>>(P, views, nviews, err);
    else k_check_columns<GEOM_CONE, MODEL_CUBIC><<<grid, 256, 0, st>>>(P, views, nviews, err);
  } else {
    if (P.model == MODEL_TABLE) k_check_columns<GEOM_PARALLEL, MODEL_TABLE><<<grid, 256, 0, st>>>(P, views, nviews, err);
    else k_check_columns<GEOM_PARALLEL, MODEL_CUBIC><<<grid, 256, 0, st>>>(P, views, nviews, err);
  }
  return cudaGetLastError();
}

cudaError_t launch_fwd3d(const Fwd3DLaunch &L, cudaStream_t st)
{
  // factorised views: the band kernels of proj3d_fast.cu (both models; the
  // table model with its exact FP64 per-voxel axes)
  if (L.band_rows > 0) return launch_fwd3d_fast(L, st);
  if (L.P.geom == GEOM_CONE)
    return L.P.model == MODEL_TABLE ? launch_fwd<GEOM_CONE, MODEL_TABLE>(L, st)
                                    : launch_fwd<GEOM_CONE, MODEL_CUBIC>(L, st);
  return L.P.model == MODEL_TABLE ? launch_fwd<GEOM_PARALLEL, MODEL_TABLE>(L, st)
                                  : launch_fwd<GEOM_PARALLEL, MODEL_CUBIC>(L, st);
}

cudaError_t launch_back3d(const Back3DLaunch &L, cudaStream_t st)
{
  // factorised views: the column kernels of proj3d_fast.cu (both models;
  // the table model with its exact FP64 per-voxel axes)
  if (L.factorized) return launch_back3d_fast(L, st);
  if (L.P.geom == GEOM_CONE)
    return L.P.model == MODEL_TABLE ? launch_back<GEOM_CONE, MODEL_TABLE>(L, st)
                                    : launch_back<GEOM_CONE, MODEL_CUBIC>(L, st);
  return L.P.model == MODEL_TABLE ? launch_back<GEOM_PARALLEL, MODEL_TABLE>(L, st)
                                  : launch_back<GEOM_PARALLEL, MODEL_CUBIC>(L, st);
}

}  // namespace trtt
