// proj3d_fast.cu -- per-view 3D projector pair for column-factorised views
// (circular orbits), both footprint models.
//
// Direct: one CTA per (band of detector rows, view) accumulates the band in
// shared memory; its warps pull 32-column chunks, build each hit column's
// u-profile and spread it over the band rows with the column's v-weights
// (fast3d_items.cuh: band_item for the closed-form cubic footprint, two
// voxels per lane with packed FP32x2 arithmetic; band_item_table for the
// tabulated footprint, with the reference's exact FP64 per-voxel axes).
// Every detector cell has one owning CTA: no global atomics.  Transpose:
// one warp per voxel column and k range gathers, view by view, through the
// column's v-collapsed detector profile (column_item), Kahan-compensated,
// atomic-free.  Both directions call the same footprint functions, so the
// pair is an exact adjoint up to FP32 summation.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "fast3d_items.cuh"
#include "kernels.h"

namespace trtt {

// ---------------------------------------------------------------------------
// Direct projector
// ---------------------------------------------------------------------------
// One CTA: detector rows [v0, v1) of view blockIdx.y, band in shared memory
// (band item of the model), written back once.
template <int GEOM, int MODEL>
__device__ __forceinline__ void band_cta(const Params3D &P, const View3D *__restrict__ views,
                                         const float *__restrict__ vol, long gate_stride,
                                         float *__restrict__ sino, long sino_view_stride,
                                         int band_rows, int *__restrict__ err, int lock_spread)
{
  extern __shared__ float sm[];
  __shared__ View3D sV;
  __shared__ int s_next;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv;
  float *acc = sm;
  float *prof = sm + band_rows * nu + warp * nu;
  float *wv = sm + band_rows * nu + nwarps * nu + warp * band_rows;
  int *locks = reinterpret_cast<int *>(sm + band_rows * nu + nwarps * nu + nwarps * band_rows);
  const int vi = blockIdx.y;
  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] =
        reinterpret_cast<const double *>(views + vi)[threadIdx.x];
  if (threadIdx.x == 0) s_next = 0;
  const int v0 = blockIdx.x * band_rows;
  const int v1 = min(v0 + band_rows, nv);
  for (int t = threadIdx.x; t < band_rows * nu; t += blockDim.x) acc[t] = 0.f;
  for (int t = threadIdx.x; t < band_rows; t += blockDim.x) locks[t] = 0;
  for (int t = lane; t < nu; t += 32) prof[t] = 0.f;
  __syncthreads();
  if constexpr (MODEL == MODEL_TABLE)
    band_item_table<GEOM>(P, sV, vol, gate_stride, v0, v1, acc, prof, wv, locks, &s_next, err,
                          lock_spread != 0);
  else
    band_item<GEOM>(P, sV, vol, gate_stride, v0, v1, band_rows, acc, prof, wv, locks, &s_next, err,
                    lock_spread != 0);
  __syncthreads();
  float *out = sino + (long)vi * sino_view_stride;
  const int nrow = v1 - v0;
  for (int t = threadIdx.x; t < nrow * nu; t += blockDim.x) {
    const int r = t / nu, u = t - r * nu;
    out[(long)(v0 + r) * nu + u] += acc[t];
  }
}

template <int GEOM>
__global__ void __launch_bounds__(512)
k_fwd3d_band_fast(const Params3D P, const View3D *__restrict__ views,
                  const float *__restrict__ vol, long gate_stride, float *__restrict__ sino,
                  long sino_view_stride, int band_rows, int *__restrict__ err, int lock_spread)
{
  band_cta<GEOM, MODEL_CUBIC>(P, views, vol, gate_stride, sino, sino_view_stride, band_rows, err,
                              lock_spread);
}

// Table model: the FP64 per-voxel axes; MINB CTAs per SM (register budget).
template <int GEOM, int MINB>
__global__ void __launch_bounds__(512, MINB)
k_fwd3d_band_table(const Params3D P, const View3D *__restrict__ views,
                   const float *__restrict__ vol, long gate_stride, float *__restrict__ sino,
                   long sino_view_stride, int band_rows, int *__restrict__ err, int lock_spread)
{
  band_cta<GEOM, MODEL_TABLE>(P, views, vol, gate_stride, sino, sino_view_stride, band_rows, err,
                              lock_spread);
}

// ---------------------------------------------------------------------------
// Direct projector, column pairs.  Same band decomposition as
// k_fwd3d_band_fast, but a warp takes the hits of a chunk two at a time
// (neighbouring columns along x, whose footprints nearly coincide), builds
// both profiles and spreads w1(r) P1[u] + w2(r) P2[u] over the union of
// their rows and cells: one shared-memory atomic per cell of the union
// instead of one per cell of each column.
// ---------------------------------------------------------------------------
template <int GEOM>
__global__ void __launch_bounds__(512)
k_fwd3d_band_pair(const Params3D P, const View3D *__restrict__ views,
                  const float *__restrict__ vol, long gate_stride, float *__restrict__ sino,
                  long sino_view_stride, int band_rows, int *__restrict__ err)
{
  extern __shared__ float sm[];
  __shared__ View3D sV;
  __shared__ int s_next;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv;
  float *acc = sm;
  float *prof1 = sm + band_rows * nu + warp * 2 * nu;
  float *prof2 = prof1 + nu;
  float *wv1 = sm + band_rows * nu + nwarps * 2 * nu + warp * 2 * band_rows;
  float *wv2 = wv1 + band_rows;
  const int vi = blockIdx.y;
  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] =
        reinterpret_cast<const double *>(views + vi)[threadIdx.x];
  if (threadIdx.x == 0) s_next = 0;
  const int v0 = blockIdx.x * band_rows;
  const int v1 = min(v0 + band_rows, nv);
  for (int t = threadIdx.x; t < band_rows * nu; t += blockDim.x) acc[t] = 0.f;
  for (int t = lane; t < 2 * nu; t += 32) prof1[t] = 0.f;
  for (int t = lane; t < 2 * band_rows; t += 32) wv1[t] = 0.f;
  __syncthreads();
  const View3D &V = sV;
  const int ncols = P.nx * P.ny;
  const int nchunks = (ncols + 31) >> 5;

  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(&s_next, 1);
    chunk = __shfl_sync(FULLM, chunk, 0);
    if (chunk >= nchunks) break;
    const int mycol = (chunk << 5) + lane;
    ColGeo<MODEL_CUBIC> c;
    bool hit = false;
    if (mycol < ncols) {
      column_geo<GEOM, MODEL_CUBIC>(P, V, mycol % P.nx, mycol / P.nx, 0, c);
      if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      hit = !c.bad && c.vax.n > 0 && c.vax.lo + c.vax.n > v0 && c.vax.lo < v1;
    }
    unsigned mask = __ballot_sync(FULLM, hit);
    while (mask) {
      const int s1 = __ffs(mask) - 1;
      mask &= mask - 1;
      const int s2 = mask ? __ffs(mask) - 1 : -1;
      if (s2 >= 0) mask &= mask - 1;
      const ColGeo<MODEL_CUBIC> c1 = shfl_colc(c, s1);
      const ColGeo<MODEL_CUBIC> c2 = shfl_colc(c, s2 >= 0 ? s2 : s1);
      // rows of each column inside the band, and their union
      const int rb1 = max(c1.vax.lo, v0), re1 = min(c1.vax.lo + c1.vax.n, v1);
      int rb = rb1, re = re1, rb2 = 0, re2 = 0;
      if (s2 >= 0) {
        rb2 = max(c2.vax.lo, v0);
        re2 = min(c2.vax.lo + c2.vax.n, v1);
        rb = min(rb, rb2);
        re = max(re, re2);
      }
      for (int r = rb + lane; r < re; r += 32) {
        wv1[r - v0] = (r >= rb1 && r < re1) ? axis_weight<MODEL_CUBIC>(c1.vax, r - c1.vax.lo, P) : 0.f;
        wv2[r - v0] = (s2 >= 0 && r >= rb2 && r < re2) ? axis_weight<MODEL_CUBIC>(c2.vax, r - c2.vax.lo, P) : 0.f;
      }
      int lo1, hi1, lo2 = INT_MAX, hi2 = INT_MIN;
      column_profile<GEOM>(P, V, vol, gate_stride, c1, (chunk << 5) + s1, prof1, lane, lo1, hi1);
      if (s2 >= 0) column_profile<GEOM>(P, V, vol, gate_stride, c2, (chunk << 5) + s2, prof2, lane, lo2, hi2);
      const int lo = min(lo1, lo2), hi = max(hi1, hi2);
      __syncwarp();
      if (lo < hi) {
        for (int r = rb; r < re; ++r) {
          const float w1 = wv1[r - v0], w2 = wv2[r - v0];
          float *row = acc + (r - v0) * nu;
          for (int u = lo + lane; u < hi; u += 32) atomicAdd(row + u, fmaf(w2, prof2[u], w1 * prof1[u]));
        }
        __syncwarp();
        for (int u = lo + lane; u < hi; u += 32) {
          prof1[u] = 0.f;
          prof2[u] = 0.f;
        }
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
// Direct projector, atomic-free band accumulation ("pull").
//
// A CTA owns 32 detector rows of one view; each of its 16 warps owns two of
// them (warp w: rows w and w+16) and each lane UC consecutive cells of both
// rows, accumulated in registers.  Work proceeds in batches: every warp takes
// its next column that touches the band, builds the column's u-profile
// P[u] (sum over the column's voxels of rho * x * u-weight) in its shared
// row and publishes the column's weights on the 32 band rows; after a
// barrier every thread adds w(row) * P[u] of the 16 profiles into the cells
// it owns.  Each detector cell has one owner, so no atomics are needed
// outside the per-warp profiles and the summation order is fixed.
// ---------------------------------------------------------------------------
template <int GEOM, int UC>
__global__ void __launch_bounds__(512, 1)
k_fwd3d_pull(const Params3D P, const View3D *__restrict__ views,
             const float *__restrict__ vol, long gate_stride, float *__restrict__ sino,
             long sino_view_stride, int *__restrict__ err)
{
  constexpr int NW = 16, BR = 32, ROW = 32 * UC;
  extern __shared__ float sm[];
  float *prof_all = sm;               // NW rows of ROW floats
  float *Wb = sm + NW * ROW;          // Wb[c * BR + r]: weight of warp c's column on band row r
  int *rng = reinterpret_cast<int *>(Wb + NW * BR);  // [lo, hi) of each warp's profile
  __shared__ View3D sV;
  __shared__ int s_next;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv, nz = P.nz;
  float *prof = prof_all + warp * ROW;
  const int vi = blockIdx.y;
  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] =
        reinterpret_cast<const double *>(views + vi)[threadIdx.x];
  if (threadIdx.x == 0) s_next = 0;
  const int v0 = blockIdx.x * BR;
  const int v1 = min(v0 + BR, nv);
  for (int t = lane; t < ROW; t += 32) prof[t] = 0.f;
  __syncthreads();
  const View3D &V = sV;
  const int ncols = P.nx * P.ny;
  const int nchunks = (ncols + 31) >> 5;
  float acc0[UC], acc1[UC];
#pragma unroll
  for (int q = 0; q < UC; ++q) {
    acc0[q] = 0.f;
    acc1[q] = 0.f;
  }
  // per-warp cursor over 32-column candidate chunks
  unsigned mask = 0;
  int chunk = -1;
  bool exhausted = false;
  ColGeo<MODEL_CUBIC> c;
  c.vax.n = 0;
  for (;;) {
    int col = -1;
    ColGeo<MODEL_CUBIC> cc;
    while (!exhausted) {
      if (mask == 0) {
        int ch = 0;
        if (lane == 0) ch = atomicAdd(&s_next, 1);
        chunk = __shfl_sync(FULLM, ch, 0);
        if (chunk >= nchunks) {
          exhausted = true;
          break;
        }
        const int mycol = (chunk << 5) + lane;
        bool hit = false;
        if (mycol < ncols) {
          column_geo<GEOM, MODEL_CUBIC>(P, V, mycol % P.nx, mycol / P.nx, 0, c);
          if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
          hit = !c.bad && c.vax.n > 0 && c.vax.lo + c.vax.n > v0 && c.vax.lo < v1;
        }
        mask = __ballot_sync(FULLM, hit);
        continue;
      }
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      cc = shfl_colc(c, src);
      col = (chunk << 5) + src;
      break;
    }
    const bool have = col >= 0;
    int lo = INT_MAX, hi = INT_MIN;
    // band weights of this warp's column (0 outside its footprint)
    {
      float w = 0.f;
      const int r = v0 + lane;
      if (have && lane < BR && r < v1 && r >= cc.vax.lo && r < cc.vax.lo + cc.vax.n)
        w = axis_weight<MODEL_CUBIC>(cc.vax, r - cc.vax.lo, P);
      if (lane < BR) Wb[warp * BR + lane] = w;
    }
    if (have) {
      const long cbase = (long)col * nz;
      for (int k0 = lane; k0 < nz; k0 += 64) {
        const int k1 = k0 + 32;
        const float x0 = vox_val(vol, gate_stride, V, cbase + k0);
        const float x1 = (k1 < nz) ? vox_val(vol, gate_stride, V, cbase + k1) : 0.0f;
        if (x0 == 0.0f && x1 == 0.0f) continue;
        UPair up;
        voxel_u_pair<GEOM>(P, V, cc, k0, k1, up);
        if (x0 == 0.0f) up.n0 = 0;
        if (x1 == 0.0f) up.n1 = 0;
        const int L = max(up.n0, up.n1);
        if (L <= 0) continue;
        const float2 xr = mul2(make_float2(x0, x1), up.rho);
        float2 Fp = first_edge_prim2(up);
        float2 lf = f2(1.0f);
        for (int l = 0; l < L; ++l) {
          const float2 F = cubic_prim2(fma2(lf, up.inc, up.start));
          const float2 w = mul2(add2(F, make_float2(-Fp.x, -Fp.y)), xr);
          if (l < up.n0) atomicAdd(prof + up.lo0 + l, w.x);
          if (l < up.n1) atomicAdd(prof + up.lo1 + l, w.y);
          Fp = F;
          lf = add2(lf, f2(1.0f));
        }
        if (up.n0 > 0) {
          lo = min(lo, up.lo0);
          hi = max(hi, up.lo0 + up.n0);
        }
        if (up.n1 > 0) {
          lo = min(lo, up.lo1);
          hi = max(hi, up.lo1 + up.n1);
        }
      }
      lo = __reduce_min_sync(FULLM, lo);
      hi = __reduce_max_sync(FULLM, hi);
    }
    if (lane == 0) {
      rng[2 * warp] = lo;
      rng[2 * warp + 1] = hi;
    }
    if (!__syncthreads_or(have ? 1 : 0)) break;
    // pull: cells (row warp, row warp+16) x [ub, ub+UC)
    const int ub = lane * UC;
#pragma unroll 1
    for (int cw = 0; cw < NW; ++cw) {
      const float w0 = Wb[cw * BR + warp];
      const float w1 = Wb[cw * BR + warp + NW];
      if (w0 == 0.f && w1 == 0.f) continue;
      const int clo = rng[2 * cw], chi = rng[2 * cw + 1];
      if (ub + UC <= clo || ub >= chi) continue;
      const float4 *pc = reinterpret_cast<const float4 *>(prof_all + cw * ROW + ub);
#pragma unroll
      for (int q = 0; q < UC / 4; ++q) {
        const float4 p4 = pc[q];
        acc0[4 * q + 0] = fmaf(w0, p4.x, acc0[4 * q + 0]);
        acc0[4 * q + 1] = fmaf(w0, p4.y, acc0[4 * q + 1]);
        acc0[4 * q + 2] = fmaf(w0, p4.z, acc0[4 * q + 2]);
        acc0[4 * q + 3] = fmaf(w0, p4.w, acc0[4 * q + 3]);
        acc1[4 * q + 0] = fmaf(w1, p4.x, acc1[4 * q + 0]);
        acc1[4 * q + 1] = fmaf(w1, p4.y, acc1[4 * q + 1]);
        acc1[4 * q + 2] = fmaf(w1, p4.z, acc1[4 * q + 2]);
        acc1[4 * q + 3] = fmaf(w1, p4.w, acc1[4 * q + 3]);
      }
    }
    __syncthreads();
    if (have && lo < hi)
      for (int u = lo + lane; u < hi; u += 32) prof[u] = 0.f;
    __syncwarp();
  }
  // write the owned cells back (each cell has exactly one owner)
  float *out = sino + (long)vi * sino_view_stride;
  const int ub = lane * UC;
  const int r0 = v0 + warp, r1 = v0 + warp + NW;
#pragma unroll
  for (int q = 0; q < UC; ++q) {
    const int u = ub + q;
    if (u < nu) {
      if (r0 < v1) out[(long)r0 * nu + u] += acc0[q];
      if (r1 < v1) out[(long)r1 * nu + u] += acc1[q];
    }
  }
}

// ---------------------------------------------------------------------------
// Transpose
// ---------------------------------------------------------------------------
template <int GEOM, int KP, int MODEL>
__global__ void __launch_bounds__(256)
k_back3d_col_fast(const Params3D P, const View3D *__restrict__ views,
                  const int *__restrict__ gate_ptr, const GateEntry *__restrict__ entries,
                  int view_lo, int view_hi, const float *__restrict__ sino,
                  long sino_view_stride, float *__restrict__ vol, long gate_stride,
                  int *__restrict__ err, int vec4)
{
  extern __shared__ float sm[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5;
  const int ncols = P.nx * P.ny;
  const int col = blockIdx.x * nwarps + warp;
  if (col >= ncols) return;
  const int gate = blockIdx.z;
  column_item<GEOM, KP, LoadNC, MODEL>(P, views, entries, gate_ptr[gate], gate_ptr[gate + 1], view_lo,
                                view_hi, sino, sino_view_stride, vol, gate_stride, col,
                                blockIdx.y * (64 * KP), gate, sm + warp * P.nu, err, vec4 != 0);
}

// Transpose of a gated scan, all gates in one pass over the views: one warp
// per (column, range of 64 KP voxels); each view's contribution goes to its
// two gates (pairs[view]).  Shared memory per warp: the profile row and the
// per-gate sums and compensations (back_gates_row floats).
template <int GEOM, int KP, int MODEL>
__global__ void __launch_bounds__(256)
k_back3d_col_gates(const Params3D P, const View3D *__restrict__ views,
                   const GatePair *__restrict__ pairs, int view_lo, int view_hi,
                   const float *__restrict__ sino, long sino_view_stride, float *__restrict__ vol,
                   long gate_stride, int ngates, int *__restrict__ err, int vec4)
{
  extern __shared__ __align__(16) float sm_g[];
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5;
  const int ncols = P.nx * P.ny;
  const int col = blockIdx.x * nwarps + warp;
  if (col >= ncols) return;
  float *row = sm_g + (size_t)warp * back_gates_row(P.nu, ngates, KP);
  float *sacc = row + ((P.nu + 3) & ~3), *scmp = sacc + ngates * 64 * KP;
  column_item_gates<GEOM, KP, LoadNC, MODEL>(P, views, pairs, view_lo, view_hi, sino, sino_view_stride, vol,
                                      gate_stride, ngates, col, blockIdx.y * (64 * KP), row, sacc, scmp,
                                      err, vec4 != 0);
}

// ---------------------------------------------------------------------------
// Launchers (cubic model, factorised views)
// ---------------------------------------------------------------------------
template <int GEOM, int UC>
static cudaError_t fwd_pull(const Fwd3DLaunch &L, cudaStream_t st)
{
  dim3 grid((L.P.nv + 31) / 32, L.nviews);
  const size_t smem = sizeof(float) * (16 * 32 * UC + 16 * 32) + sizeof(int) * 32;
  auto kern = k_fwd3d_pull<GEOM, UC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, 512, smem, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino, L.sino_view_stride,
                                L.err);
  return cudaGetLastError();
}

template <int GEOM, int MODEL, int MINB = 1>
static cudaError_t fwd_band(const Fwd3DLaunch &L, cudaStream_t st)
{
  dim3 grid((L.P.nv + L.band_rows - 1) / L.band_rows, L.nviews);
  const size_t smem = band_fast_smem(L.P.nu, L.band_rows, L.warps);
  auto kern = MODEL == MODEL_TABLE ? k_fwd3d_band_table<GEOM, MINB> : k_fwd3d_band_fast<GEOM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, L.warps * 32, smem, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino,
                                        L.sino_view_stride, L.band_rows, L.err,
                                        band_lock_spread(L.P) ? 1 : 0);
  return cudaGetLastError();
}

template <int GEOM>
static cudaError_t fwd_fast(const Fwd3DLaunch &L, cudaStream_t st)
{
  if (L.P.model == MODEL_TABLE) {
    // Two 16-warp CTAs per SM (64 registers per thread) only where their
    // shared memory leaves the cumulative table (read through L1 at random
    // slots) room in the SM's 256 KB of L1 and shared memory; else one
    // (up to 128 registers).  With the table evicted from L1 every edge
    // lookup goes to L2.
    const size_t smem = band_fast_smem(L.P.nu, L.band_rows, L.warps);
    const size_t table = sizeof(double) * (size_t)L.P.size + 16u * 1024u;
    const bool two = L.warps == 16 && 2 * (smem + 1024) <= 228u * 1024u &&
                     2 * (smem + 1024) + table <= 256u * 1024u;
    return two ? fwd_band<GEOM, MODEL_TABLE, 2>(L, st) : fwd_band<GEOM, MODEL_TABLE, 1>(L, st);
  }
  if (L.pull) {
    if (L.P.nu <= 128) return fwd_pull<GEOM, 4>(L, st);
    if (L.P.nu <= 256) return fwd_pull<GEOM, 8>(L, st);
    if (L.P.nu <= 512) return fwd_pull<GEOM, 16>(L, st);
  }
  dim3 grid((L.P.nv + L.band_rows - 1) / L.band_rows, L.nviews);
  if (L.cols == 2) {
    const size_t smem = sizeof(float) * ((size_t)L.band_rows * L.P.nu + 2 * (size_t)L.warps * L.P.nu +
                                         2 * (size_t)L.warps * L.band_rows);
    auto kern = k_fwd3d_band_pair<GEOM>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, L.warps * 32, smem, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino,
                                          L.sino_view_stride, L.band_rows, L.err);
    return cudaGetLastError();
  }
  return fwd_band<GEOM, MODEL_CUBIC>(L, st);
}

template <int GEOM, int KP, int MODEL>
static cudaError_t back_fast_kp(const Back3DLaunch &L, cudaStream_t st)
{
  const int warps = 8;
  const int ncols = L.P.nx * L.P.ny;
  const int kblocks = (L.P.nz + 64 * KP - 1) / (64 * KP);
  // 16-byte profile loads: rows of nu % 4 == 0 floats in 16-byte aligned images
  const int vec4 = (L.P.nu % 4 == 0 && L.sino_view_stride % 4 == 0 &&
                    ((uintptr_t)L.sino & 15) == 0) ? 1 : 0;
  const size_t smem_gates = sizeof(float) * (size_t)warps * back_gates_row(L.P.nu, L.ngates, KP);
  if (L.pairs && L.ngates > 1 && smem_gates <= 160u * 1024u) {
    dim3 grid((ncols + warps - 1) / warps, kblocks);
    auto kern = k_back3d_col_gates<GEOM, KP, MODEL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_gates);
    if (e != cudaSuccess) return e;
    kern<<<grid, warps * 32, smem_gates, st>>>(L.P, L.views, L.pairs, L.view_lo, L.view_hi, L.sino,
                                               L.sino_view_stride, L.vol, L.gate_stride, L.ngates,
                                               L.err, vec4);
    return cudaGetLastError();
  }
  dim3 grid((ncols + warps - 1) / warps, kblocks, L.ngates);
  const size_t smem = sizeof(float) * (size_t)warps * L.P.nu;
  auto kern = k_back3d_col_fast<GEOM, KP, MODEL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, warps * 32, smem, st>>>(L.P, L.views, L.gate_ptr, L.entries, L.view_lo, L.view_hi,
                                      L.sino, L.sino_view_stride, L.vol, L.gate_stride, L.err, vec4);
  return cudaGetLastError();
}

// Voxel pairs per lane by column length: 64 voxels (1), 128 (2), more (4;
// the table model, whose per-voxel axes are FP64, at most 2), so that short
// columns do not carry idle pairs.
template <int GEOM, int MODEL>
static cudaError_t back_fast(const Back3DLaunch &L, cudaStream_t st)
{
  if (L.P.nz <= 64) return back_fast_kp<GEOM, 1, MODEL>(L, st);
  if (L.P.nz <= 128 || MODEL == MODEL_TABLE) return back_fast_kp<GEOM, 2, MODEL>(L, st);
  return back_fast_kp<GEOM, MODEL == MODEL_TABLE ? 2 : 4, MODEL>(L, st);
}

cudaError_t launch_fwd3d_fast(const Fwd3DLaunch &L, cudaStream_t st)
{
  if (L.tc && L.P.model == MODEL_CUBIC) return launch_fwd3d_tc(L, st);
  return L.P.geom == GEOM_CONE ? fwd_fast<GEOM_CONE>(L, st) : fwd_fast<GEOM_PARALLEL>(L, st);
}

cudaError_t launch_back3d_fast(const Back3DLaunch &L, cudaStream_t st)
{
  if (L.P.model == MODEL_TABLE)
    return L.P.geom == GEOM_CONE ? back_fast<GEOM_CONE, MODEL_TABLE>(L, st)
                                 : back_fast<GEOM_PARALLEL, MODEL_TABLE>(L, st);
  return L.P.geom == GEOM_CONE ? back_fast<GEOM_CONE, MODEL_CUBIC>(L, st)
                               : back_fast<GEOM_PARALLEL, MODEL_CUBIC>(L, st);
}

size_t band_fast_smem(int nu, int band_rows, int warps)
{
  // band, one profile and one row-weight list per warp, one lock per row
  return sizeof(float) * ((size_t)band_rows * nu + (size_t)warps * nu + (size_t)warps * band_rows +
                          (size_t)band_rows);
}

}  // namespace trtt
