// proj3d.cu -- sm_100a kernels of the 3D B-spline projector pair
// (trtt_PB3D/CB3D, table and closed-form cubic footprints, and the per-gate
// projections of the 4D path).
//
// Direct projector (voxel-driven, detector-row bands in shared memory):
//   grid (bands, views).  A CTA owns `band_rows` full detector rows of one
//   view in shared memory.  Its warps pull 32-column chunks of the volume
//   from a shared counter, test each column's transaxial footprint against
//   the band (one lane per column), and for every hit the whole warp walks
//   the column (one voxel per lane, coalesced along k): the u-weights of
//   each voxel are accumulated into a per-warp row profile P[u]
//   (shared-memory atomics, ~5 voxels per cell), then P is spread into the
//   band rows with the column's v-weights.  The band is written back once
//   (each detector cell has exactly one owning CTA: no global atomics).
//
// Transpose (voxel-driven gather, atomic-free):
//   one warp per voxel column.  For each view the lanes first form the
//   column's v-collapsed detector profile Q[u] = sum_v wv(v) pix[v,u]
//   (shared memory), then every voxel gathers sum_u wu(u) Q[u] with its own
//   u-weights.  Views are accumulated per voxel in registers with Kahan
//   compensation; the volume is read and written once per launch.
//
// Both use the weights of geom3d.cuh, so the pair is an exact adjoint up to
// FP32 rounding.  Views whose transaxial footprint depends on k (general
// xforms) use the per-voxel kernels at the end of this file.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "geom3d.cuh"
#include "kernels.h"

namespace trtt {

static constexpr unsigned FULL = 0xffffffffu;

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

// Broadcast a column state from lane `src`.
template <int MODEL>
__device__ __forceinline__ ColGeo<MODEL> shfl_col(const ColGeo<MODEL> &c, int src)
{
  ColGeo<MODEL> r;
  r.vax.lo = __shfl_sync(FULL, c.vax.lo, src);
  r.vax.n = __shfl_sync(FULL, c.vax.n, src);
  r.vax.start = __shfl_sync(FULL, c.vax.start, src);
  r.vax.inc = __shfl_sync(FULL, c.vax.inc, src);
  r.bad = __shfl_sync(FULL, c.bad, src);
  r.q = __shfl_sync(FULL, c.q, src);
  r.magn = __shfl_sync(FULL, c.magn, src);
  r.delta_v = __shfl_sync(FULL, c.delta_v, src);
  r.vca8sqr = __shfl_sync(FULL, c.vca8sqr, src);
  r.nyj = __shfl_sync(FULL, c.nyj, src);
  r.nxi = __shfl_sync(FULL, c.nxi, src);
  r.A = __shfl_sync(FULL, c.A, src);
  r.B = __shfl_sync(FULL, c.B, src);
  r.h_u0m = __shfl_sync(FULL, c.h_u0m, src);
  r.rho0c = __shfl_sync(FULL, c.rho0c, src);
  r.inv_den = __shfl_sync(FULL, c.inv_den, src);
  return r;
}

// ---------------------------------------------------------------------------
// Direct projector, factorised views: detector-row bands.
// ---------------------------------------------------------------------------
template <int GEOM, int MODEL>
__global__ void __launch_bounds__(512)
k_fwd3d_band(const Params3D P, const View3D *__restrict__ views,
             const float *__restrict__ vol, long gate_stride,
             float *__restrict__ sino, long sino_view_stride, int band_rows,
             int *__restrict__ err)
{
  extern __shared__ float sm[];
  __shared__ View3D sV;
  __shared__ int s_next;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv, nz = P.nz;
  float *acc = sm;
  float *prof = sm + band_rows * nu + warp * nu;
  float *wv = sm + band_rows * nu + nwarps * nu + warp * band_rows;
  const int vi = blockIdx.y;
  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] =
        reinterpret_cast<const double *>(views + vi)[threadIdx.x];
  if (threadIdx.x == 0) s_next = 0;
  const int v0 = blockIdx.x * band_rows;
  const int v1 = min(v0 + band_rows, nv);
  for (int t = threadIdx.x; t < band_rows * nu; t += blockDim.x) acc[t] = 0.f;
  for (int t = lane; t < nu; t += 32) prof[t] = 0.f;
  __syncthreads();
  const View3D &V = sV;
  const int ncols = P.nx * P.ny;
  const int nchunks = (ncols + 31) >> 5;

  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(&s_next, 1);
    chunk = __shfl_sync(FULL, chunk, 0);
    if (chunk >= nchunks) break;
    const int mycol = (chunk << 5) + lane;
    ColGeo<MODEL> c;
    bool hit = false;
    if (mycol < ncols) {
      const int i = mycol % P.nx, j = mycol / P.nx;
      column_geo<GEOM, MODEL>(P, V, i, j, 0, c);
      if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      const int vr = c.vax.lo + c.vax.n;
      hit = !c.bad && c.vax.n > 0 && vr > v0 && c.vax.lo < v1;
    }
    unsigned mask = __ballot_sync(FULL, hit);
    while (mask) {
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      const ColGeo<MODEL> cc = shfl_col<MODEL>(c, src);
      const int col = (chunk << 5) + src;
      const int vl = cc.vax.lo, vr = cc.vax.lo + cc.vax.n;
      const int rb = max(vl, v0), re = min(vr, v1), nr = re - rb;
      for (int r = lane; r < nr; r += 32) wv[r] = axis_weight<MODEL>(cc.vax, rb - vl + r, P);
      // u-profile of the column
      int lo = INT_MAX, hi = INT_MIN;
      const long cbase = (long)col * nz;
      for (int k = lane; k < nz; k += 32) {
        const float x = voxel_value(vol, gate_stride, V, cbase + k);
        if (x == 0.0f) continue;
        typename AxisOf<MODEL>::type ax;
        float rho0;
        if (!voxel_u<GEOM, MODEL>(P, V, cc, k, ax, rho0)) continue;
        const float xr = x * rho0;
        if constexpr (MODEL == MODEL_TABLE) {
          double p0 = edge_table(ax, 0, P.cum, P.last);
          for (int l = 0; l < ax.n; ++l) {
            double p1 = edge_table(ax, l + 1, P.cum, P.last);
            atomicAdd(prof + ax.lo + l, (float)(p1 - p0) * xr);
            p0 = p1;
          }
        } else {
          float p0 = edge_cubic(ax, 0);
          for (int l = 0; l < ax.n; ++l) {
            float p1 = edge_cubic(ax, l + 1);
            atomicAdd(prof + ax.lo + l, (p1 - p0) * xr);
            p0 = p1;
          }
        }
        lo = min(lo, ax.lo);
        hi = max(hi, ax.lo + ax.n);
      }
      lo = __reduce_min_sync(FULL, lo);
      hi = __reduce_max_sync(FULL, hi);
      __syncwarp();
      if (lo < hi) {
        for (int r = 0; r < nr; ++r) {
          const float w = wv[r];
          float *row = acc + (rb - v0 + r) * nu;
          for (int u = lo + lane; u < hi; u += 32) atomicAdd(row + u, w * prof[u]);
        }
        __syncwarp();
        for (int u = lo + lane; u < hi; u += 32) prof[u] = 0.f;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  float *out = sino + (long)vi * sino_view_stride;
  const int nrow = v1 - v0;
  for (int t = threadIdx.x; t < nrow * nu; t += blockDim.x) {
    const int r = t / nu, u = t - r * nu;
    out[(long)(v0 + r) * nu + u] += acc[t];
  }
}

// ---------------------------------------------------------------------------
// Transpose, factorised views: one warp per column, gather per voxel.
// Entries (view, weight) come from a per-gate list (CSR: gate_ptr[g] ..
// gate_ptr[g+1]); plain 3D uses one gate and weight 1.
// ---------------------------------------------------------------------------
template <int GEOM, int MODEL, int KR>
__global__ void __launch_bounds__(256)
k_back3d_col(const Params3D P, const View3D *__restrict__ views,
             const int *__restrict__ gate_ptr, const GateEntry *__restrict__ entries,
             int view_lo, int view_hi,
             const float *__restrict__ sino, long sino_view_stride,
             float *__restrict__ vol, long gate_stride, int *__restrict__ err)
{
  extern __shared__ float sm[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nz = P.nz;
  const int ncols = P.nx * P.ny;
  const int col = blockIdx.x * nwarps + warp;
  if (col >= ncols) return;
  float *Q = sm + warp * nu;
  float *wv = sm + nwarps * nu + warp * 64;
  const int i = col % P.nx, j = col / P.nx;
  const int kbase = blockIdx.y * (32 * KR);
  const int gate = blockIdx.z;
  const int e0 = gate_ptr[gate], e1 = gate_ptr[gate + 1];
  Kahan acc[KR];

  for (int eb = e0; eb < e1; eb += 32) {
    // lanes evaluate the column state of 32 consecutive entries at once
    const int me = eb + lane;
    ColGeo<MODEL> mine;
    int myview = 0;
    float myw = 0.f;
    const GateEntry ge = (me < e1) ? entries[me] : GateEntry{-1, 0.f};
    if (ge.view >= view_lo && ge.view < view_hi) {
      myview = ge.view;
      myw = ge.w;
      column_geo<GEOM, MODEL>(P, views[myview], i, j, 0, mine);
      if (mine.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
    } else {
      mine.vax.n = 0;
      mine.bad = 1;
    }
    const int cnt = min(32, e1 - eb);
    for (int s = 0; s < cnt; ++s) {
      const int nvx = __shfl_sync(FULL, mine.vax.n, s);
      const int bd = __shfl_sync(FULL, mine.bad, s);
      if (bd || nvx <= 0) continue;
      const ColGeo<MODEL> cc = shfl_col<MODEL>(mine, s);
      const int view = __shfl_sync(FULL, myview, s);
      const float wgt = __shfl_sync(FULL, myw, s);
      const View3D &V = views[view];
      const int npv = cc.vax.n;
      // u footprints of this lane's voxels
      typename AxisOf<MODEL>::type ax[KR];
      float rho[KR];
      int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
      for (int r = 0; r < KR; ++r) {
        const int k = kbase + lane + 32 * r;
        ax[r].n = 0;
        rho[r] = 0.f;
        if (k < nz && voxel_u<GEOM, MODEL>(P, V, cc, k, ax[r], rho[r])) {
          lo = min(lo, ax[r].lo);
          hi = max(hi, ax[r].lo + ax[r].n);
        }
      }
      lo = __reduce_min_sync(FULL, lo);
      hi = __reduce_max_sync(FULL, hi);
      if (lo >= hi) continue;
      // v weights, then the v-collapsed profile Q[u] over [lo, hi)
      for (int m0 = 0; m0 < npv; m0 += 64) {
        const int mn = min(64, npv - m0);
        for (int m = lane; m < mn; m += 32) wv[m] = axis_weight<MODEL>(cc.vax, m0 + m, P);
        __syncwarp();
        const float *img = sino + (long)(view - view_lo) * sino_view_stride + (long)(cc.vax.lo + m0) * nu;
        for (int u = lo + lane; u < hi; u += 32) {
          float s0 = (m0 == 0) ? 0.f : Q[u];
          for (int m = 0; m < mn; ++m) s0 = fmaf(wv[m], __ldg(img + (long)m * nu + u), s0);
          Q[u] = s0;
        }
        __syncwarp();
      }
      // per-voxel gather
#pragma unroll
      for (int r = 0; r < KR; ++r) {
        if (ax[r].n > 0) {
          float s0 = 0.f;
          if constexpr (MODEL == MODEL_TABLE) {
            double p0 = edge_table(ax[r], 0, P.cum, P.last);
            for (int l = 0; l < ax[r].n; ++l) {
              double p1 = edge_table(ax[r], l + 1, P.cum, P.last);
              s0 = fmaf((float)(p1 - p0), Q[ax[r].lo + l], s0);
              p0 = p1;
            }
          } else {
            float p0 = edge_cubic(ax[r], 0);
            for (int l = 0; l < ax[r].n; ++l) {
              float p1 = edge_cubic(ax[r], l + 1);
              s0 = fmaf(p1 - p0, Q[ax[r].lo + l], s0);
              p0 = p1;
            }
          }
          acc[r].add(wgt * rho[r] * s0);
        }
      }
      __syncwarp();
    }
  }
  float *dst = vol + (long)gate * gate_stride + (long)col * nz;
#pragma unroll
  for (int r = 0; r < KR; ++r) {
    const int k = kbase + lane + 32 * r;
    if (k < nz) dst[k] += acc[r].value();
  }
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
  if (L.band_rows > 0) {
    dim3 grid((L.P.nv + L.band_rows - 1) / L.band_rows, L.nviews);
    const size_t smem = sizeof(float) * ((size_t)L.band_rows * L.P.nu +
                                         (size_t)L.warps * L.P.nu +
                                         (size_t)L.warps * L.band_rows);
    auto kern = k_fwd3d_band<GEOM, MODEL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, L.warps * 32, smem, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino,
                                          L.sino_view_stride, L.band_rows, L.err);
  } else {
    const long nvox = (long)L.P.nx * L.P.ny * L.P.nz;
    dim3 grid((unsigned)((nvox + 255) / 256), L.nviews);
    k_fwd3d_vox<GEOM, MODEL><<<grid, 256, 0, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino,
                                                  L.sino_view_stride, L.err);
  }
  return cudaGetLastError();
}

template <int GEOM, int MODEL>
static cudaError_t launch_back(const Back3DLaunch &L, cudaStream_t st)
{
  const int ncols = L.P.nx * L.P.ny;
  if (L.factorized) {
    constexpr int KR = 8;
    const int warps = 8;
    dim3 grid((ncols + warps - 1) / warps, (L.P.nz + 32 * KR - 1) / (32 * KR), L.ngates);
    const size_t smem = sizeof(float) * ((size_t)warps * L.P.nu + (size_t)warps * 64);
    auto kern = k_back3d_col<GEOM, MODEL, KR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, warps * 32, smem, st>>>(L.P, L.views, L.gate_ptr, L.entries, L.view_lo, L.view_hi, L.sino,
                                        L.sino_view_stride, L.vol, L.gate_stride, L.err);
  } else {
    const long nvox = (long)ncols * L.P.nz;
    dim3 grid((unsigned)((nvox + 255) / 256), 1, L.ngates);
    k_back3d_vox<GEOM, MODEL><<<grid, 256, 0, st>>>(L.P, L.views, L.gate_ptr, L.entries, L.view_lo, L.view_hi, L.sino,
                                                   L.sino_view_stride, L.vol, L.gate_stride, L.err);
  }
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
  if (L.P.model == MODEL_CUBIC && L.band_rows > 0) return launch_fwd3d_fast(L, st);
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
