// fast3d_items.cuh -- the work items of the closed-form (cubic) projector
// pair on column-factorised views, shared by the per-view grid kernels
// (proj3d_fast.cu) and the persistent 4D kernel (persist4d.cu):
//
//  * band item (direct): one CTA accumulates, for one view, the detector
//    rows [v0, v1) in shared memory: warps pull 32-column chunks from a
//    shared counter, build each hit column's u-profile (two voxels per lane,
//    packed FP32x2) and spread it over the band rows with the column's
//    v-weights, one row at a time under a row lock;
//  * column item (transpose): one warp gathers, for one voxel column and
//    k range, the contributions of every (view, weight) entry of a gate: per
//    view the v-collapsed profile Q[u] = sum_v w(v) pix[v][u] is built in
//    registers and each voxel pair gathers it with its u-weights; views are
//    accumulated with packed Kahan compensation.
#pragma once

#include <climits>

#include "fast3d.cuh"
#include "kernels.h"

namespace trtt {

static constexpr int SPREAD_CHUNKS = 16;  // footprints up to 512 cells wide spread from registers
static constexpr int TABLE_LMAX = 10;     // table model: footprints up to 10 cells from registers

// True when floor(uc_k - hs_k), the first cell of voxel k's u-footprint
// before any clamp, strictly increases or decreases along the column: the
// voxels of one warp step then write distinct cells at every footprint
// offset l, so a warp can update its profile with plain loads and stores.
// |d uc/dk| = |B|; hs = hs0 h_u0 magn delta_u varies by at most
// hs0 h_u0m |B| max|uc - a12| u_scl^2 inv_den per voxel.
template <int GEOM, int MODEL = MODEL_CUBIC>
__device__ __forceinline__ bool column_monotone(const Params3D &P, const View3D &V,
                                                const ColGeo<MODEL> &c)
{
  const double b = fabs(c.B);
  if constexpr (GEOM == GEOM_CONE) {
    const double ua = c.A, ub = fma(c.B, (double)(P.nz - 1), c.A);
    const double um = fmax(fabs(ua - V.a12), fabs(ub - V.a12));
    const double dhs = P.hs0 * (double)c.h_u0m * b * um * P.u_scl * P.u_scl * (double)c.inv_den;
    return b - dhs >= 1.002;
  } else {
    return b >= 1.002;
  }
}

__device__ __forceinline__ unsigned long long timer_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Exclusive use of one band row by a warp (lane 0 takes the lock, the warp
// then updates the row with plain loads and stores).  The wait is bounded:
// past 2 s the warp sets TRTT_ERR_STALL and skips the row.  A holder
// releases after a few hundred cycles, so the limit is never reached in a
// correct run.
__device__ __forceinline__ bool row_lock(int *lock, int *err)
{
  int got = 1;
  if ((threadIdx.x & 31) == 0) {
    if (atomicCAS(lock, 0, 1) != 0) {
      const unsigned long long t0 = timer_ns();
      while (atomicCAS(lock, 0, 1) != 0) {
        if (timer_ns() - t0 > 2000000000ull) {
          atomicOr(err, TRTT_ERR_STALL);
          got = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence_block();
  }
  got = __shfl_sync(FULLM, got, 0);
  __syncwarp();
  return got != 0;
}

__device__ __forceinline__ void row_unlock(int *lock)
{
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    __threadfence_block();
    atomicExch(lock, 0);
  }
}


// Spread of a warp's column profile over the band: acc[rb - v0 + r][u] +=
// wv[r] * prof[u] for the nr rows r and the cells [lo, hi) (lo, hi: the
// lane's own range, reduced here over the warp); the profile is cleared on
// the way.  Modes as in band_item.  All lanes call it.
__device__ __forceinline__ void band_spread(int lo, int hi, int rb, int v0, int nr, int nu,
                                            float *acc, float *prof, const float *wv, int *locks,
                                            int *__restrict__ err, bool lock_spread)
{
  const int lane = threadIdx.x & 31;
  lo = __reduce_min_sync(FULLM, lo);
  hi = __reduce_max_sync(FULLM, hi);
  __syncwarp();
  if (lo < hi && hi - lo <= 32 * SPREAD_CHUNKS) {
    // profile read once into registers (and cleared), then the rows
    // one at a time
    float pv[SPREAD_CHUNKS];
#pragma unroll
    for (int q = 0; q < SPREAD_CHUNKS; ++q) {
      const int u = lo + lane + 32 * q;
      pv[q] = 0.f;
      if (u < hi) {
        pv[q] = prof[u];
        prof[u] = 0.f;
      }
    }
    for (int r = 0; r < nr; ++r) {
      const float w = wv[r];
      const int row = rb - v0 + r;
      float *rowp = acc + row * nu;
      if (lock_spread) {
        if (!row_lock(locks + row, err)) continue;
#pragma unroll
        for (int q = 0; q < SPREAD_CHUNKS; ++q) {
          const int u = lo + lane + 32 * q;
          if (u < hi) rowp[u] = fmaf(w, pv[q], rowp[u]);
        }
        row_unlock(locks + row);
      } else {
#pragma unroll
        for (int q = 0; q < SPREAD_CHUNKS; ++q) {
          const int u = lo + lane + 32 * q;
          if (u < hi) atomicAdd(rowp + u, w * pv[q]);
        }
      }
    }
  } else if (lo < hi) {
    for (int r = 0; r < nr; ++r) {
      const float w = wv[r];
      const int row = rb - v0 + r;
      float *rowp = acc + row * nu;
      if (lock_spread) {
        if (!row_lock(locks + row, err)) continue;
        for (int u = lo + lane; u < hi; u += 32) rowp[u] = fmaf(w, prof[u], rowp[u]);
        row_unlock(locks + row);
      } else {
        for (int u = lo + lane; u < hi; u += 32) atomicAdd(rowp + u, w * prof[u]);
      }
    }
    __syncwarp();
    for (int u = lo + lane; u < hi; u += 32) prof[u] = 0.f;
  }
  __syncwarp();
}

// Band item.  acc: band_rows x nu floats (zeroed by the caller), prof: this
// warp's nu-float profile (zero on entry and on exit), wv: this warp's
// band_rows floats, locks: band_rows ints (zero, shared by the CTA), s_next:
// the CTA's chunk counter (0 on entry), lock_spread: spread mode (below,
// the same for the whole CTA).  All threads of the CTA call it; it returns
// without a final barrier.
//
// Profile: where floor(uc - hs) is strictly monotone along the column
// (column_monotone) the 64 voxels of a warp step write 64 distinct cells at
// every footprint offset, so each voxel walks its footprint from the
// unclamped first cell (primitive 0 there) with plain loads and stores,
// steps ordered by __syncwarp; other columns use shared atomics.  Spread:
// with lock_spread the warp takes each band row exclusively (row_lock) and
// adds w(v) P[u] with plain loads and stores, else one shared atomic per
// cell and row.  Shared float atomics are compare-and-swap loops, so the
// locks pay on long rows (long voxel columns); on short ones the warps
// meet on the same rows and the atomics are faster (band_lock_spread).
template <int GEOM>
__device__ __forceinline__ void band_item(const Params3D &P, const View3D &V,
                                          const float *__restrict__ vol, long gate_stride, int v0,
                                          int v1, int band_rows, float *acc, float *prof, float *wv,
                                          int *locks, int *s_next, int *__restrict__ err,
                                          bool lock_spread)
{
  const int lane = threadIdx.x & 31;
  const int nu = P.nu, nz = P.nz;
  const int ncols = P.nx * P.ny;
  const int nchunks = (ncols + 31) >> 5;
  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(s_next, 1);
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
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      const ColGeo<MODEL_CUBIC> cc = shfl_colc(c, src);
      const int col = (chunk << 5) + src;
      const int vl = cc.vax.lo, vr = cc.vax.lo + cc.vax.n;
      const int rb = max(vl, v0), re = min(vr, v1), nr = re - rb;
      for (int r = lane; r < nr; r += 32) wv[r] = axis_weight<MODEL_CUBIC>(cc.vax, rb - vl + r, P);
      int lo = INT_MAX, hi = INT_MIN;
      const long cbase = (long)col * nz;
      if (column_monotone<GEOM>(P, V, cc)) {
        for (int kb = 0; kb < nz; kb += 64) {
          const int k0 = kb + lane, k1 = k0 + 32;
          const float x0 = (k0 < nz) ? vox_val(vol, gate_stride, V, cbase + k0) : 0.0f;
          const float x1 = (k1 < nz) ? vox_val(vol, gate_stride, V, cbase + k1) : 0.0f;
          if (!__any_sync(FULLM, x0 != 0.0f || x1 != 0.0f)) continue;
          UPair up;
          voxel_u_pair<GEOM>(P, V, cc, k0, k1, up);
          if (x0 == 0.0f) up.n0 = 0;
          if (x1 == 0.0f) up.n1 = 0;
          const double uc0 = fma(cc.B, (double)k0, cc.A), uc1 = fma(cc.B, (double)k1, cc.A);
          const float2 hsv = mul2(make_float2(__frcp_rn(up.inc.x), __frcp_rn(up.inc.y)),
                                  f2((float)P.hs0));
          const int f0 = __double2int_rd(uc0 - (double)hsv.x), f1 = __double2int_rd(uc1 - (double)hsv.y);
          // the reference's first cell is f clamped to [0, nu-1]: cells left
          // of the detector are not written; a footprint that starts past it
          // (f >= nu) gives its one clamped cell weight 0 - 0 and is dropped
          const int e0 = up.n0 > 0 ? up.lo0 + up.n0 : INT_MIN;
          const int e1 = up.n1 > 0 ? up.lo1 + up.n1 : INT_MIN;
          const int L0 = (up.n0 > 0 && f0 < nu) ? max(e0 - f0, 0) : 0;
          const int L1 = (up.n1 > 0 && f1 < nu) ? max(e1 - f1, 0) : 0;
          const int Lw = __reduce_max_sync(FULLM, max(max(L0, L1), 0));
          if (Lw <= 0) continue;
          const float2 start = make_float2(fmaf((float)(f0 - up.lo0), up.inc.x, up.start.x),
                                           fmaf((float)(f1 - up.lo1), up.inc.y, up.start.y));
          const float2 xr = mul2(make_float2(x0, x1), up.rho);
          float2 Fp = f2(0.0f);
          float2 lf = f2(1.0f);
          for (int l = 0; l < Lw; ++l) {
            const float2 F = cubic_prim2(fma2(lf, up.inc, start));
            const float2 w = add2(F, make_float2(-Fp.x, -Fp.y));
            const int c0 = f0 + l, c1 = f1 + l;
            if (l < L0 && c0 >= 0) prof[c0] = fmaf(w.x, xr.x, prof[c0]);
            if (l < L1 && c1 >= 0) prof[c1] = fmaf(w.y, xr.y, prof[c1]);
            __syncwarp();
            Fp = F;
            lf = add2(lf, f2(1.0f));
          }
          if (L0 > 0 && e0 > max(f0, 0)) {
            lo = min(lo, max(f0, 0));
            hi = max(hi, e0);
          }
          if (L1 > 0 && e1 > max(f1, 0)) {
            lo = min(lo, max(f1, 0));
            hi = max(hi, e1);
          }
        }
      } else {
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
      }
      band_spread(lo, hi, rb, v0, nr, nu, acc, prof, wv, locks, err, lock_spread);
    }
  }
}

// Detector loads of the column item: read-only data (__ldg) in the grid
// kernels; data written earlier in the same launch (L2, coherent) in the
// persistent kernel.
struct LoadNC {
  __device__ __forceinline__ static float ld(const float *p) { return __ldg(p); }
  __device__ __forceinline__ static float4 ld4(const float4 *p) { return __ldg(p); }
};
struct LoadCG {
  __device__ __forceinline__ static float ld(const float *p) { return __ldcg(p); }
  __device__ __forceinline__ static float4 ld4(const float4 *p) { return __ldcg(p); }
};

// Column state of lane `src`, for either footprint model.
template <int MODEL>
__device__ __forceinline__ ColGeo<MODEL> shfl_colm(const ColGeo<MODEL> &c, int src)
{
  if constexpr (MODEL == MODEL_CUBIC) {
    return shfl_colc(c, src);
  } else {
    ColGeo<MODEL> r;
    r.vax.lo = __shfl_sync(FULLM, c.vax.lo, src);
    r.vax.n = __shfl_sync(FULLM, c.vax.n, src);
    r.vax.start = __shfl_sync(FULLM, c.vax.start, src);
    r.vax.inc = __shfl_sync(FULLM, c.vax.inc, src);
    r.bad = 0;
    r.q = __shfl_sync(FULLM, c.q, src);
    r.magn = __shfl_sync(FULLM, c.magn, src);
    r.delta_v = __shfl_sync(FULLM, c.delta_v, src);
    r.vca8sqr = __shfl_sync(FULLM, c.vca8sqr, src);
    r.nyj = __shfl_sync(FULLM, c.nyj, src);
    r.nxi = __shfl_sync(FULLM, c.nxi, src);
    return r;
  }
}

// Per-voxel u-footprints of a lane's voxels k0, k1 (either model): the
// closed form evaluates both with packed FP32 (UPair); the table model
// keeps the reference's exact FP64 axes (voxel_u), so that every table slot
// is the reference's own.
template <int MODEL> struct VoxPair;
template <> struct VoxPair<MODEL_CUBIC> {
  UPair up;
};
template <> struct VoxPair<MODEL_TABLE> {
  AxisTable ax0, ax1;
  float rho0, rho1;
};

// Band item of the table model (direct, column-factorised views): the
// decomposition of band_item with the reference's exact FP64 per-voxel
// axes (voxel_u<GEOM, MODEL_TABLE>) and FP64 table edges, so every table
// slot is the reference's own.  Lane j takes voxel kb + j of a warp step
// (FP64 axes leave nothing to pack).  Profile: on a monotone column
// (column_monotone) the 32 voxels of a step have distinct first cells
// unless a first cell was clamped to the detector's first or last cell, so
// a step without such a cell writes distinct cells at every footprint
// offset and updates the profile with plain loads and stores (offsets
// ordered by __syncwarp); other steps use shared atomics.  Footprints of
// up to TABLE_LMAX cells load their edges together into registers first.
// Spread: band_spread.  Same arguments and contract as band_item.
template <int GEOM>
__device__ __forceinline__ void band_item_table(const Params3D &P, const View3D &V,
                                                const float *__restrict__ vol, long gate_stride,
                                                int v0, int v1, float *acc, float *prof, float *wv,
                                                int *locks, int *s_next, int *__restrict__ err,
                                                bool lock_spread)
{
  const int lane = threadIdx.x & 31;
  const int nu = P.nu, nz = P.nz;
  const int ncols = P.nx * P.ny;
  const int nchunks = (ncols + 31) >> 5;
  const double *__restrict__ cum = P.cum;
  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(s_next, 1);
    chunk = __shfl_sync(FULLM, chunk, 0);
    if (chunk >= nchunks) break;
    const int mycol = (chunk << 5) + lane;
    ColGeo<MODEL_TABLE> c;
    bool hit = false;
    int my_mono = 0;
    if (mycol < ncols) {
      column_geo<GEOM, MODEL_TABLE>(P, V, mycol % P.nx, mycol / P.nx, 0, c);
      if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      hit = !c.bad && c.vax.n > 0 && c.vax.lo + c.vax.n > v0 && c.vax.lo < v1;
      if (hit) my_mono = column_monotone<GEOM, MODEL_TABLE>(P, V, c) ? 1 : 0;
    }
    unsigned mask = __ballot_sync(FULLM, hit);
    while (mask) {
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      const ColGeo<MODEL_TABLE> cc = shfl_colm<MODEL_TABLE>(c, src);
      const bool mono = __shfl_sync(FULLM, my_mono, src) != 0;
      const int col = (chunk << 5) + src;
      const int vl = cc.vax.lo, vr = cc.vax.lo + cc.vax.n;
      const int rb = max(vl, v0), re = min(vr, v1), nr = re - rb;
      for (int r = lane; r < nr; r += 32) wv[r] = axis_weight<MODEL_TABLE>(cc.vax, rb - vl + r, P);
      int lo = INT_MAX, hi = INT_MIN;
      const long cbase = (long)col * nz;
      for (int kb = 0; kb < nz; kb += 32) {
        const int k = kb + lane;
        const float x = (k < nz) ? vox_val(vol, gate_stride, V, cbase + k) : 0.0f;
        if (!__any_sync(FULLM, x != 0.0f)) continue;
        AxisTable ax{};
        float rho0 = 0.f;
        int n = 0;
        if (x != 0.0f && voxel_u<GEOM, MODEL_TABLE>(P, V, cc, k, ax, rho0)) n = ax.n;
        const float xr = x * rho0;
        const bool edge = n > 0 && (ax.lo == 0 || ax.lo == nu - 1);
        const int Lw = __reduce_max_sync(FULLM, n);
        if (Lw <= TABLE_LMAX) {
          // the footprint's weights first: its n + 1 table edges are
          // independent loads, issued together
          float w[TABLE_LMAX];
          {
            double e[TABLE_LMAX + 1];
#pragma unroll
            for (int l = 0; l <= TABLE_LMAX; ++l) e[l] = (l <= n) ? edge_table(ax, l, cum, P.last) : 0.0;
#pragma unroll
            for (int l = 0; l < TABLE_LMAX; ++l) w[l] = (float)(e[l + 1] - e[l]) * xr;
          }
          if (mono && !__any_sync(FULLM, edge)) {
#pragma unroll
            for (int l = 0; l < TABLE_LMAX; ++l) {
              if (l < Lw) {
                if (l < n) prof[ax.lo + l] += w[l];
                __syncwarp();
              }
            }
          } else {
#pragma unroll
            for (int l = 0; l < TABLE_LMAX; ++l)
              if (l < n) atomicAdd(prof + ax.lo + l, w[l]);
          }
        } else {
          double p0 = n > 0 ? edge_table(ax, 0, cum, P.last) : 0.0;
          for (int l = 0; l < n; ++l) {
            const double p1 = edge_table(ax, l + 1, cum, P.last);
            atomicAdd(prof + ax.lo + l, (float)(p1 - p0) * xr);
            p0 = p1;
          }
        }
        if (n > 0) {
          lo = min(lo, ax.lo);
          hi = max(hi, ax.lo + n);
        }
      }
      band_spread(lo, hi, rb, v0, nr, nu, acc, prof, wv, locks, err, lock_spread);
    }
  }
}

// One view's contribution to the voxels kbase + lane + 64 p (+32), p < KP,
// of column (i, j): term[p] = rho * sum_u w(u) Q[u] for the lane's two
// voxels, with Q[u] = sum_v wv(v) img[v][u] the column's v-collapsed profile
// of the view's image `img0`, built in this warp's nu-float row Q.  cc is
// the column's geometry in the view.  Returns false (term untouched, Q not
// used) when the footprints of the warp's voxels miss the detector.  vec4:
// nu % 4 == 0 and 16-byte aligned images (16-byte loads).  All lanes call it.
template <int GEOM, int KP, class LD, int MODEL = MODEL_CUBIC>
__device__ __forceinline__ bool view_gather(const Params3D &P, const View3D &V,
                                            const ColGeo<MODEL> &cc, int kbase,
                                            const float *img0, float *Q, bool vec4,
                                            float2 (&term)[KP])
{
  const int lane = threadIdx.x & 31;
  const int nu = P.nu, nz = P.nz;
  VoxPair<MODEL> vp[KP];
  int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    const int k0 = kbase + lane + 64 * p, k1 = k0 + 32;
    int lo0 = 0, n0 = 0, lo1 = 0, n1 = 0;
    if constexpr (MODEL == MODEL_CUBIC) {
      UPair &up = vp[p].up;
      voxel_u_pair<GEOM>(P, V, cc, k0, k1, up);
      if (k0 >= nz) up.n0 = 0;
      if (k1 >= nz) up.n1 = 0;
      lo0 = up.lo0; n0 = up.n0; lo1 = up.lo1; n1 = up.n1;
    } else {
      VoxPair<MODEL_TABLE> &t = vp[p];
      t.ax0.n = 0;
      t.ax1.n = 0;
      if (!(k0 < nz && voxel_u<GEOM, MODEL_TABLE>(P, V, cc, k0, t.ax0, t.rho0))) t.ax0.n = 0;
      if (!(k1 < nz && voxel_u<GEOM, MODEL_TABLE>(P, V, cc, k1, t.ax1, t.rho1))) t.ax1.n = 0;
      lo0 = t.ax0.lo; n0 = t.ax0.n; lo1 = t.ax1.lo; n1 = t.ax1.n;
    }
    if (n0 > 0) {
      lo = min(lo, lo0);
      hi = max(hi, lo0 + n0);
    }
    if (n1 > 0) {
      lo = min(lo, lo1);
      hi = max(hi, lo1 + n1);
    }
  }
  lo = __reduce_min_sync(FULLM, lo);
  hi = __reduce_max_sync(FULLM, hi);
  if (lo >= hi) return false;
  // v-collapsed profile Q[u] = sum_v wv(v) pix[v][u], u in [lo, hi).
  // Each lane keeps up to QC cells of Q in registers (u = lo + lane + 32c)
  // and walks the footprint rows; the QC loads of a row are independent,
  // so a warp keeps many loads in flight.
  const int npv = cc.vax.n;
  if (vec4) {
    // cover [lo & ~3, hi rounded up to 4): 16-byte loads, packed FMAs
    constexpr int QV = 4;
    const int a0 = lo & ~3, a1 = (hi + 3) & ~3;
    for (int ub = a0; ub < a1; ub += 128 * QV) {
      float4 q[QV];
#pragma unroll
      for (int c = 0; c < QV; ++c) q[c] = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int m0 = 0; m0 < npv; m0 += 32) {
        const int mn = min(32, npv - m0);
        const float wl = (lane < mn) ? axis_weight<MODEL>(cc.vax, m0 + lane, P) : 0.f;
        for (int m = 0; m < mn; ++m) {
          const float2 w = f2(__shfl_sync(FULLM, wl, m));
          const float4 *row =
              reinterpret_cast<const float4 *>(img0 + (long)(cc.vax.lo + m0 + m) * nu + ub + 4 * lane);
          float4 a[QV];
#pragma unroll
          for (int c = 0; c < QV; ++c)
            a[c] = (ub + 4 * lane + 128 * c < a1) ? LD::ld4(row + 32 * c) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int c = 0; c < QV; ++c) {
            const float2 l2 = fma2(w, make_float2(a[c].x, a[c].y), make_float2(q[c].x, q[c].y));
            const float2 h2 = fma2(w, make_float2(a[c].z, a[c].w), make_float2(q[c].z, q[c].w));
            q[c] = make_float4(l2.x, l2.y, h2.x, h2.y);
          }
        }
      }
#pragma unroll
      for (int c = 0; c < QV; ++c) {
        const int u = ub + 4 * lane + 128 * c;
        if (u < a1) *reinterpret_cast<float4 *>(Q + u) = q[c];
      }
    }
  } else {
    constexpr int QC = 16;
    for (int ub = lo; ub < hi; ub += 32 * QC) {
      float q[QC];
#pragma unroll
      for (int c = 0; c < QC; ++c) q[c] = 0.f;
      for (int m0 = 0; m0 < npv; m0 += 32) {
        const int mn = min(32, npv - m0);
        const float wl = (lane < mn) ? axis_weight<MODEL>(cc.vax, m0 + lane, P) : 0.f;
        for (int m = 0; m < mn; ++m) {
          const float w = __shfl_sync(FULLM, wl, m);
          const float *row = img0 + (long)(cc.vax.lo + m0 + m) * nu + ub + lane;
          float a[QC];
#pragma unroll
          for (int c = 0; c < QC; ++c) a[c] = (ub + lane + 32 * c < hi) ? LD::ld(row + 32 * c) : 0.f;
#pragma unroll
          for (int c = 0; c < QC; ++c) q[c] = fmaf(w, a[c], q[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < QC; ++c)
        if (ub + lane + 32 * c < hi) Q[ub + lane + 32 * c] = q[c];
    }
  }
  __syncwarp();
  // per-voxel gathers
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    term[p] = f2(0.f);
    if constexpr (MODEL == MODEL_CUBIC) {
      // two voxels per instruction
      const UPair &up = vp[p].up;
      const int L = max(up.n0, up.n1);
      if (L <= 0) continue;
      float2 Fp = first_edge_prim2(up);
      float2 S = f2(0.f);
      float2 lf = f2(1.0f);
      for (int l = 0; l < L; ++l) {
        const float2 F = cubic_prim2(fma2(lf, up.inc, up.start));
        const float2 w = add2(F, make_float2(-Fp.x, -Fp.y));
        const float q0 = (l < up.n0) ? Q[up.lo0 + l] : 0.0f;
        const float q1 = (l < up.n1) ? Q[up.lo1 + l] : 0.0f;
        S = fma2(w, make_float2(q0, q1), S);
        Fp = F;
        lf = add2(lf, f2(1.0f));
      }
      term[p] = mul2(up.rho, S);
    } else {
      // table edges in FP64 at the reference's positions (edge_table)
      const VoxPair<MODEL_TABLE> &t = vp[p];
      float s0 = 0.f, s1 = 0.f;
      if (t.ax0.n > 0) {
        double p0 = edge_table(t.ax0, 0, P.cum, P.last);
        for (int l = 0; l < t.ax0.n; ++l) {
          const double p1 = edge_table(t.ax0, l + 1, P.cum, P.last);
          s0 = fmaf((float)(p1 - p0), Q[t.ax0.lo + l], s0);
          p0 = p1;
        }
      }
      if (t.ax1.n > 0) {
        double p0 = edge_table(t.ax1, 0, P.cum, P.last);
        for (int l = 0; l < t.ax1.n; ++l) {
          const double p1 = edge_table(t.ax1, l + 1, P.cum, P.last);
          s1 = fmaf((float)(p1 - p0), Q[t.ax1.lo + l], s1);
          p0 = p1;
        }
      }
      term[p] = make_float2(t.rho0 * s0, t.rho1 * s1);
    }
  }
  __syncwarp();  // Q is free for the next view
  return true;
}

// Packed Kahan step: acc += term with compensation cmp.
__device__ __forceinline__ void kahan2(float2 &acc, float2 &cmp, float2 term)
{
  const float2 y = add2(term, make_float2(-cmp.x, -cmp.y));
  const float2 t = add2(acc, y);
  cmp = add2(add2(t, make_float2(-acc.x, -acc.y)), make_float2(-y.x, -y.y));
  acc = t;
}

// Column item.  One warp: column col = (i, j), voxels kbase + lane + 64 p
// (+32), p < KP, gate `gate`; the entries [e0, e1) of the gate's list with
// views in [view_lo, view_hi) (images at sino[view - view_lo]).  Q: this
// warp's nu floats.  vec4: nu % 4 == 0 and 16-byte aligned images (the
// profile is then built from 16-byte loads).  Adds the result into vol (one
// owner per voxel).
template <int GEOM, int KP, class LD, int MODEL = MODEL_CUBIC>
__device__ __forceinline__ void column_item(const Params3D &P, const View3D *__restrict__ views,
                                            const GateEntry *__restrict__ entries, int e0, int e1,
                                            int view_lo, int view_hi, const float *sino,
                                            long sino_view_stride, float *__restrict__ vol,
                                            long gate_stride, int col, int kbase, int gate, float *Q,
                                            int *__restrict__ err, bool vec4 = false)
{
  const int lane = threadIdx.x & 31;
  const int nz = P.nz;
  const int i = col % P.nx, j = col / P.nx;
  float2 acc[KP], cmp[KP];
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    acc[p] = f2(0.f);
    cmp[p] = f2(0.f);
  }
  for (int eb = e0; eb < e1; eb += 32) {
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
      const int nvx = __shfl_sync(FULLM, mine.vax.n, s);
      const int bd = __shfl_sync(FULLM, mine.bad, s);
      if (bd || nvx <= 0) continue;
      const ColGeo<MODEL> cc = shfl_colm<MODEL>(mine, s);
      const int view = __shfl_sync(FULLM, myview, s);
      const float wgt = __shfl_sync(FULLM, myw, s);
      float2 term[KP];
      if (!view_gather<GEOM, KP, LD, MODEL>(P, views[view], cc, kbase,
                                     sino + (long)(view - view_lo) * sino_view_stride, Q, vec4, term))
        continue;
#pragma unroll
      for (int p = 0; p < KP; ++p) kahan2(acc[p], cmp[p], mul2(term[p], f2(wgt)));
    }
  }
  float *dst = vol + (long)gate * gate_stride + (long)col * nz;
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    const int k0 = kbase + lane + 64 * p, k1 = k0 + 32;
    if (k0 < nz) dst[k0] += acc[p].x - cmp[p].x;
    if (k1 < nz) dst[k1] += acc[p].y - cmp[p].y;
  }
}

// Column item over all gates at once.  One warp: column col, voxels
// kbase + lane + 64 p (+32), p < KP; every view of [view_lo, view_hi) once
// (images at sino[view - view_lo]), its contribution added with weight
// pairs[view].w0 into gate pairs[view].g0 and with w1 into g1 (g1 < 0:
// none).  Per-gate sums with Kahan compensation live in this warp's shared
// rows sacc / scmp ([ngates][64 KP] floats each; lane-private entries);
// the result is added into vol (one owner per voxel and gate).
template <int GEOM, int KP, class LD, int MODEL = MODEL_CUBIC>
__device__ __forceinline__ void column_item_gates(const Params3D &P, const View3D *__restrict__ views,
                                                  const GatePair *__restrict__ pairs, int view_lo,
                                                  int view_hi, const float *sino, long sino_view_stride,
                                                  float *__restrict__ vol, long gate_stride, int ngates,
                                                  int col, int kbase, float *Q, float *sacc, float *scmp,
                                                  int *__restrict__ err, bool vec4 = false)
{
  const int lane = threadIdx.x & 31;
  const int nz = P.nz;
  const int i = col % P.nx, j = col / P.nx;
  constexpr int W = 64 * KP;
  for (int t = lane; t < ngates * W; t += 32) {
    sacc[t] = 0.f;
    scmp[t] = 0.f;
  }
  __syncwarp();
  for (int vb = view_lo; vb < view_hi; vb += 32) {
    const int myview = vb + lane;
    ColGeo<MODEL> mine;
    if (myview < view_hi) {
      column_geo<GEOM, MODEL>(P, views[myview], i, j, 0, mine);
      if (mine.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
    } else {
      mine.vax.n = 0;
      mine.bad = 1;
    }
    const int cnt = min(32, view_hi - vb);
    for (int s = 0; s < cnt; ++s) {
      const int nvx = __shfl_sync(FULLM, mine.vax.n, s);
      const int bd = __shfl_sync(FULLM, mine.bad, s);
      if (bd || nvx <= 0) continue;
      const ColGeo<MODEL> cc = shfl_colm<MODEL>(mine, s);
      const int view = vb + s;
      float2 term[KP];
      if (!view_gather<GEOM, KP, LD, MODEL>(P, views[view], cc, kbase,
                                     sino + (long)(view - view_lo) * sino_view_stride, Q, vec4, term))
        continue;
      const GatePair gp = pairs[view];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int g = h ? gp.g1 : gp.g0;
        const float wg = h ? gp.w1 : gp.w0;
        if (g < 0) continue;
        float *a = sacc + g * W, *c = scmp + g * W;
#pragma unroll
        for (int p = 0; p < KP; ++p) {
          const int v0 = 64 * p + lane, v1 = v0 + 32;
          float2 acc = make_float2(a[v0], a[v1]), cmp = make_float2(c[v0], c[v1]);
          kahan2(acc, cmp, mul2(term[p], f2(wg)));
          a[v0] = acc.x;
          a[v1] = acc.y;
          c[v0] = cmp.x;
          c[v1] = cmp.y;
        }
      }
    }
  }
  for (int g = 0; g < ngates; ++g) {
    float *dst = vol + (long)g * gate_stride + (long)col * nz;
    const float *a = sacc + g * W, *c = scmp + g * W;
#pragma unroll
    for (int p = 0; p < KP; ++p) {
      const int k0 = kbase + lane + 64 * p, k1 = k0 + 32;
      const int v0 = 64 * p + lane, v1 = v0 + 32;
      if (k0 < nz) dst[k0] += a[v0] - c[v0];
      if (k1 < nz) dst[k1] += a[v1] - c[v1];
    }
  }
  __syncwarp();
}

}  // namespace trtt
