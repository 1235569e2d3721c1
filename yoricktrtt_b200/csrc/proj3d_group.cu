// proj3d_group.cu -- closed-form (cubic) 3D projector pair over groups of
// views related by turns of the volume grid, for column-factorised views.
//
// A circular orbit about the z axis with 4N views over 2 pi sees the grid of
// a square volume turned by a quarter turn every N views: the view at
// theta + m pi/2 projects voxel column c exactly as the view at theta
// projects column R^m(c), R(i, j) = (n-1-j, i) (see find_view_groups in
// host3d.h).  The footprint arithmetic -- the column geometry, the per-voxel
// u-footprints and the B-spline primitives, which is where the projector
// spends its instructions -- is therefore evaluated once per group of G = 4
// views (quarter turns), 2 (half turns) or 1 and applied to the G voxel
// columns it serves.  Results equal the per-view kernels' up to FP32
// summation order (the member views' coefficients agree with the turned
// ones to FP64 rounding).
//
// Direct (k_fwd3d_group): one CTA per (group, detector-row band, u tile).
// The CTA keeps the band of every member view in shared memory (G x R rows
// x U cells); warps take 32-column chunks, build for each hit column the G
// member profiles P_m[u] = sum_k rho_k x_m(k) w_k(u) in warp-private
// shared rows (the weights w_k(u) computed once for the G members) and
// spread them over the band rows with the column's v-weights.  Every
// detector cell belongs to exactly one CTA: no global atomics.
//
// Transpose (k_back3d_group): one warp per orbit {g, R g, R^2 g, R^3 g} of
// columns (G members) and k range.  For each group the warp evaluates the
// footprints of the G orbit columns at the group's first view once, builds
// the v-collapsed detector profiles Q_m[u] = sum_v w(v) y_m[v][u] of every
// member view and gathers them into the G columns' voxel accumulators
// (registers, packed Kahan): atomic-free, the exact adjoint of the direct
// kernel (same device functions).
#include <cuda_runtime.h>

#include <climits>

#include "fast3d_items.cuh"
#include "kernels.h"

namespace trtt {

namespace {

// R^t(i, j) with R(i, j) = (n-1-j, i); the half turn also on nx != ny.
__device__ __forceinline__ void turn_col(int i, int j, int t, int nx, int ny, int &oi, int &oj)
{
  t &= 3;
  if (t == 0) {
    oi = i;
    oj = j;
  } else if (t == 1) {
    oi = nx - 1 - j;
    oj = i;
  } else if (t == 2) {
    oi = nx - 1 - i;
    oj = ny - 1 - j;
  } else {
    oi = j;
    oj = ny - 1 - i;
  }
}

// Turn of member m of a group of G views (G = 4: m quarter turns; G = 2:
// the half turn).
template <int G> __host__ __device__ constexpr int member_turn(int m)
{
  return G == 4 ? m : (G == 2 ? 2 * m : 0);
}

// Conservative half support (in cells) of the u-footprints of a column:
// hs0 * h_u0 * magn * delta_u at the column's extreme u positions, plus one.
template <int GEOM>
__device__ __forceinline__ double column_u_halfwidth(const Params3D &P, const View3D &V,
                                                     const ColGeo<MODEL_CUBIC> &c)
{
  if constexpr (GEOM == GEOM_CONE) {
    const double ua = c.A, ub = fma(c.B, (double)(P.nz - 1), c.A);
    const double da = (ua - V.a12) * P.u_scl, db = (ub - V.a12) * P.u_scl;
    const double d2 = fmax(da * da, db * db);
    return P.hs0 * (double)c.h_u0m * sqrt(1.0 + d2 * (double)c.inv_den) * 1.0001 + 1.0;
  } else {
    return V.p_hs_u + 1.0;
  }
}

// Voxel range [klo, khi) of a column whose u-footprints may meet cells
// [u0, u1) (with `hsm` the column's conservative half support).
__device__ __forceinline__ void column_k_range(const ColGeo<MODEL_CUBIC> &c, double hsm, int u0,
                                               int u1, int nz, int &klo, int &khi)
{
  const double lo_u = (double)u0 - 1.0 - hsm, hi_u = (double)u1 + 1.0 + hsm;
  if (!(fabs(c.B) > 1e-300)) {
    // u position independent of k: all voxels or none
    const bool in = c.A > lo_u && c.A < hi_u;
    klo = 0;
    khi = in ? nz : 0;
    return;
  }
  double ka = (lo_u - c.A) / c.B, kb = (hi_u - c.A) / c.B;
  if (ka > kb) {
    const double t = ka;
    ka = kb;
    kb = t;
  }
  ka = fmin(fmax(floor(ka), 0.0), (double)nz);
  kb = fmin(fmax(ceil(kb) + 1.0, 0.0), (double)nz);
  klo = (int)ka;
  khi = (int)kb;
}

// cell[m] += w.x * xa[m] + w.y * xc[m] for the G interleaved member slots
// of one profile cell (the two voxels of a lane).
template <int G>
__device__ __forceinline__ void cell_fma2(float *cell, float2 w, const float (&xa)[G], const float (&xc)[G])
{
  if constexpr (G == 4) {
    float4 *q = reinterpret_cast<float4 *>(cell);
    float4 v = *q;
    v.x = fmaf(w.y, xc[0], fmaf(w.x, xa[0], v.x));
    v.y = fmaf(w.y, xc[1], fmaf(w.x, xa[1], v.y));
    v.z = fmaf(w.y, xc[2], fmaf(w.x, xa[2], v.z));
    v.w = fmaf(w.y, xc[3], fmaf(w.x, xa[3], v.w));
    *q = v;
  } else if constexpr (G == 2) {
    float2 *q = reinterpret_cast<float2 *>(cell);
    float2 v = *q;
    v.x = fmaf(w.y, xc[0], fmaf(w.x, xa[0], v.x));
    v.y = fmaf(w.y, xc[1], fmaf(w.x, xa[1], v.y));
    *q = v;
  } else {
    *cell = fmaf(w.y, xc[0], fmaf(w.x, xa[0], *cell));
  }
}

// The G member values of one interleaved profile or band cell.
template <int G> struct VecOf;
template <> struct VecOf<4> { using T = float4; };
template <> struct VecOf<2> { using T = float2; };
template <> struct VecOf<1> { using T = float; };

__device__ __forceinline__ void vec_fma(float4 &b, float w, const float4 &p)
{
  b.x = fmaf(w, p.x, b.x);
  b.y = fmaf(w, p.y, b.y);
  b.z = fmaf(w, p.z, b.z);
  b.w = fmaf(w, p.w, b.w);
}
__device__ __forceinline__ void vec_fma(float2 &b, float w, const float2 &p)
{
  b.x = fmaf(w, p.x, b.x);
  b.y = fmaf(w, p.y, b.y);
}
__device__ __forceinline__ void vec_fma(float &b, float w, const float &p) { b = fmaf(w, p, b); }

// Component M of a cell's member vector, and the vector of G values.
template <int M> __device__ __forceinline__ float comp(const float4 &v)
{
  return M == 0 ? v.x : (M == 1 ? v.y : (M == 2 ? v.z : v.w));
}
template <int M> __device__ __forceinline__ float comp(const float2 &v) { return M == 0 ? v.x : v.y; }
template <int M> __device__ __forceinline__ float comp(const float &v) { return v; }
__device__ __forceinline__ void pack(float4 &v, const float (&a)[4]) { v = make_float4(a[0], a[1], a[2], a[3]); }
__device__ __forceinline__ void pack(float2 &v, const float (&a)[2]) { v = make_float2(a[0], a[1]); }
__device__ __forceinline__ void pack(float &v, const float (&a)[1]) { v = a[0]; }

// S[m] += w * (member m of the cells a0, a1), m < G, packed over the two
// voxels of a lane.
template <int G, int M = 0>
__device__ __forceinline__ void gather_fma(float2 (&S)[G], float2 w, const typename VecOf<G>::T &a0,
                                           const typename VecOf<G>::T &a1)
{
  if constexpr (M < G) {
    S[M] = fma2(w, make_float2(comp<M>(a0), comp<M>(a1)), S[M]);
    gather_fma<G, M + 1>(S, w, a0, a1);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Direct projector over view groups
// ---------------------------------------------------------------------------
template <int GEOM, int G, bool IL, int MINB>
__global__ void __launch_bounds__(MINB == 1 ? 704 : 512, MINB)
k_fwd3d_group(const GroupFwdLaunch A)
{
  extern __shared__ __align__(16) float sm[];
  __shared__ View3D sV;
  __shared__ int s_next;
  __shared__ int s_mem[4];
  const Params3D &P = A.P;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv, nz = P.nz, nx = P.nx, ny = P.ny;
  const int R = A.band_rows, U = A.utile;
  const int band = blockIdx.x / A.usplit, ut = blockIdx.x - band * A.usplit;
  const int v0 = band * R, v1 = min(v0 + R, nv);
  const int u0 = ut * U, u1 = min(u0 + U, nu);
  const int grp = blockIdx.y;
  // member bands: [G][R][U], or [R][U][G] with interleaved profiles (IL)
  float *bands = sm;
  float *prof = sm + G * R * U + warp * G * U;          // [G][U] or [U][G], this warp
  float *wv = sm + G * R * U + nwarps * G * U + warp * R;  // [R], this warp
  int *row_locks = reinterpret_cast<int *>(sm + G * R * U + nwarps * G * U + nwarps * R);  // [R]
  const int base = A.groups[4 * grp];
  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] =
        reinterpret_cast<const double *>(A.views + base)[threadIdx.x];
  if (threadIdx.x < 4) s_mem[threadIdx.x] = A.groups[4 * grp + threadIdx.x];
  if (threadIdx.x == 0) s_next = 0;
  for (int t = threadIdx.x; t < G * R * U; t += blockDim.x) bands[t] = 0.f;
  for (int t = threadIdx.x; t < R; t += blockDim.x) row_locks[t] = 0;
  for (int t = lane; t < G * U; t += 32) prof[t] = 0.f;
  __syncthreads();
  const View3D &V = sV;
  const int ncols = nx * ny;
  const int nchunks = (ncols + 31) >> 5;

  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(&s_next, 1);
    chunk = __shfl_sync(FULLM, chunk, 0);
    if (chunk >= nchunks) break;
    const int mycol = (chunk << 5) + lane;
    ColGeo<MODEL_CUBIC> c;
    bool hit = false;
    // per column, by its own lane: the voxel range whose footprints may meet
    // the u tile and the monotone test (shuffled to the warp for each hit)
    int my_klo = 0, my_khi = nz, my_mono = 0;
    if (mycol < ncols) {
      column_geo<GEOM, MODEL_CUBIC>(P, V, mycol % nx, mycol / nx, 0, c);
      if (c.bad) atomicOr(A.err, TRTT_ERR_SOURCE_PLANE);
      hit = !c.bad && c.vax.n > 0 && c.vax.lo + c.vax.n > v0 && c.vax.lo < v1;
      if (hit && A.usplit > 1) {
        column_k_range(c, column_u_halfwidth<GEOM>(P, V, c), u0, u1, nz, my_klo, my_khi);
        hit = my_klo < my_khi;
      }
      if (IL && hit) my_mono = column_monotone<GEOM>(P, V, c) ? 1 : 0;
    }
    unsigned mask = __ballot_sync(FULLM, hit);
    while (mask) {
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      const ColGeo<MODEL_CUBIC> cc = shfl_colc(c, src);
      const int g = (chunk << 5) + src;
      const int gi = g % nx, gj = g / nx;
      // voxel columns of the members: member m sees at this footprint the
      // column R^{-t_m}(g)
      const float *colp[G];
#pragma unroll
      for (int m = 0; m < G; ++m) {
        int ci, cj;
        turn_col(gi, gj, 4 - member_turn<G>(m), nx, ny, ci, cj);
        colp[m] = A.vol + ((long)cj * nx + ci) * nz;
      }
      const int vl = cc.vax.lo, vr = cc.vax.lo + cc.vax.n;
      const int rb = max(vl, v0), re = min(vr, v1), nr = re - rb;
      for (int r = lane; r < nr; r += 32) wv[r] = axis_weight<MODEL_CUBIC>(cc.vax, rb - vl + r, P);
      const int klo = __shfl_sync(FULLM, my_klo, src), khi = __shfl_sync(FULLM, my_khi, src);
      const bool mono = __shfl_sync(FULLM, my_mono, src) != 0;
      int lo = INT_MAX, hi = INT_MIN;
      // interleaved profiles (IL): cell-major, the G member values of a cell
      // side by side; member m of cell c at prof[c * G + m], else prof[m U + c]
      const int cs = IL ? G : 1, ms = IL ? 1 : U;
      if (IL && mono) {
        // plain loads and stores.  Lane j takes the adjacent voxels 2j and
        // 2j+1 of the step (a: the one whose footprint starts lower, c: the
        // other) and walks cells f_a, f_a + 1, ... from a's unclamped first
        // cell (where the primitive is 0), adding a's weight at offset l and
        // c's at l - d (d = f_c - f_a >= 1) in one update of the cell.  The
        // first cells of the 32 lanes' pairs are at least 2 apart, so at
        // each step the warp writes 32 distinct cells; steps are ordered by
        // __syncwarp.  Cells left of the tile are not written (c >= u0).
        const int sa = cc.B > 0.0 ? 0 : 1;
        for (int kb = klo; kb < khi; kb += 64) {
          const int ka = kb + 2 * lane + sa, kc = kb + 2 * lane + (1 - sa);
          float2 x[G];
          bool any = false;
#pragma unroll
          for (int m = 0; m < G; ++m) {
            x[m].x = (ka < khi) ? __ldg(colp[m] + ka) : 0.0f;
            x[m].y = (kc < khi) ? __ldg(colp[m] + kc) : 0.0f;
            any = any || x[m].x != 0.0f || x[m].y != 0.0f;
          }
          if (!__any_sync(FULLM, any)) continue;
          UPair up;
          voxel_u_pair<GEOM>(P, V, cc, ka, kc, up);
          if (ka >= khi || !any) up.n0 = 0;
          if (kc >= khi || !any) up.n1 = 0;
          const double uc0 = fma(cc.B, (double)ka, cc.A), uc1 = fma(cc.B, (double)kc, cc.A);
          const float2 hsv = mul2(make_float2(__frcp_rn(up.inc.x), __frcp_rn(up.inc.y)),
                                  f2((float)P.hs0));
          const int f0 = __double2int_rd(uc0 - (double)hsv.x), f1 = __double2int_rd(uc1 - (double)hsv.y);
          // the reference's first cell is f clamped to [0, nu-1]: cells left
          // of the tile are not written; a footprint that starts past the
          // detector (f >= nu) gives its one clamped cell weight 0 - 0 and is
          // dropped.  Where hs rounds f one cell away from the reference's
          // lo, the cell between holds a weight below the primitive's value
          // within 1e-6 of the support end (~1e-27).
          const int e0 = up.n0 > 0 ? min(up.lo0 + up.n0, u1) : INT_MIN;
          const int e1 = up.n1 > 0 ? min(up.lo1 + up.n1, u1) : INT_MIN;
          const int L0 = (up.n0 > 0 && f0 < nu) ? max(e0 - f0, 0) : 0;
          const int L1 = (up.n1 > 0 && f1 < nu) ? max(e1 - f1, 0) : 0;
          const int d = f1 - f0;
          const int Ln = max(L0, L1 > 0 ? d + L1 : 0);
          const int Lw = __reduce_max_sync(FULLM, Ln);
          if (Lw <= 0) continue;
          const float2 start = make_float2(fmaf((float)(f0 - up.lo0), up.inc.x, up.start.x),
                                           fmaf((float)(f1 - up.lo1), up.inc.y, up.start.y));
          float xr0[G], xr1[G];
#pragma unroll
          for (int m = 0; m < G; ++m) {
            const float2 t = mul2(x[m], up.rho);
            xr0[m] = t.x;
            xr1[m] = t.y;
          }
          float2 Fp = f2(0.0f);
          float2 lf = make_float2(1.0f, (float)(1 - d));
          for (int l = 0; l < Lw; ++l) {
            const float2 F = cubic_prim2(fma2(lf, up.inc, start));
            float2 w = add2(F, make_float2(-Fp.x, -Fp.y));
            const bool on0 = l < L0, on1 = l >= d && l - d < L1;
            if (!on0) w.x = 0.0f;
            if (!on1) w.y = 0.0f;
            const int c = f0 + l;
            if ((on0 || on1) && c >= u0) cell_fma2<G>(prof + (c - u0) * G, w, xr0, xr1);
            __syncwarp();
            Fp = F;
            lf = add2(lf, f2(1.0f));
          }
          if (L0 > 0 && e0 > max(f0, u0)) {
            lo = min(lo, max(f0, u0));
            hi = max(hi, e0);
          }
          if (L1 > 0 && e1 > max(f1, u0)) {
            lo = min(lo, max(f1, u0));
            hi = max(hi, e1);
          }
        }
      } else
      for (int kb = klo; kb < khi; kb += 64) {
        const int k0 = kb + lane, k1 = k0 + 32;
        float2 x[G];
        bool any = false;
#pragma unroll
        for (int m = 0; m < G; ++m) {
          x[m].x = (k0 < khi) ? __ldg(colp[m] + k0) : 0.0f;
          x[m].y = (k1 < khi) ? __ldg(colp[m] + k1) : 0.0f;
          any = any || x[m].x != 0.0f || x[m].y != 0.0f;
        }
        if (!any) continue;
        UPair up;
        voxel_u_pair<GEOM>(P, V, cc, k0, k1, up);
        if (k0 >= khi) up.n0 = 0;
        if (k1 >= khi) up.n1 = 0;
        // clip the cell ranges to the tile; the first edge of a clipped
        // range is evaluated (it is not the support start)
        const int c0 = max(up.lo0, u0), e0 = min(up.lo0 + up.n0, u1);
        const int c1 = max(up.lo1, u0), e1 = min(up.lo1 + up.n1, u1);
        const int n0 = e0 - c0, n1 = e1 - c1;
        const int L = max(n0, n1);
        if (L <= 0) continue;
        float2 start = make_float2(fmaf((float)(c0 - up.lo0), up.inc.x, up.start.x),
                                   fmaf((float)(c1 - up.lo1), up.inc.y, up.start.y));
        float2 Fp;
        if (c0 == up.lo0 && c1 == up.lo1 && up.lo0 > 0 && up.lo1 > 0)
          Fp = f2(0.0f);
        else
          Fp = cubic_prim2(start);
        if (c0 == up.lo0 && up.lo0 > 0) Fp.x = 0.0f;
        if (c1 == up.lo1 && up.lo1 > 0) Fp.y = 0.0f;
        float2 xr[G];
#pragma unroll
        for (int m = 0; m < G; ++m) xr[m] = mul2(x[m], up.rho);
        float *p0 = prof + (c0 - u0) * cs;
        float *p1 = prof + (c1 - u0) * cs;
        float2 lf = f2(1.0f);
        for (int l = 0; l < L; ++l) {
          const float2 F = cubic_prim2(fma2(lf, up.inc, start));
          const float2 w = add2(F, make_float2(-Fp.x, -Fp.y));
#pragma unroll
          for (int m = 0; m < G; ++m) {
            const float2 p = mul2(w, xr[m]);
            if (l < n0) atomicAdd(p0 + m * ms + l * cs, p.x);
            if (l < n1) atomicAdd(p1 + m * ms + l * cs, p.y);
          }
          Fp = F;
          lf = add2(lf, f2(1.0f));
        }
        if (n0 > 0) {
          lo = min(lo, c0);
          hi = max(hi, e0);
        }
        if (n1 > 0) {
          lo = min(lo, c1);
          hi = max(hi, e1);
        }
      }
      lo = __reduce_min_sync(FULLM, lo);
      hi = __reduce_max_sync(FULLM, hi);
      __syncwarp();
      if (lo < hi) {
        constexpr int CH = 8;  // U <= 256 cells per tile
        if constexpr (IL) {
          // spread: band[r][u][m] += wv[r] * P[u][m].  The warp takes each
          // of its rows exclusively (row lock) and updates the G members of
          // a cell with one vector load and store; the profile is read once
          // into registers and cleared.
          using VecG = typename VecOf<G>::T;
          VecG pv[CH];
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            const int u = lo + lane + 32 * q;
            pv[q] = VecG{};
            if (u < hi) {
              VecG *cell = reinterpret_cast<VecG *>(prof + (u - u0) * G);
              pv[q] = *cell;
              *cell = VecG{};
            }
          }
          for (int r = 0; r < nr; ++r) {
            const float w = wv[r];
            const int row = rb - v0 + r;
            if (!row_lock(row_locks + row, A.err)) continue;
            VecG *brow = reinterpret_cast<VecG *>(bands + (size_t)row * U * G);
#pragma unroll
            for (int q = 0; q < CH; ++q) {
              const int u = lo + lane + 32 * q;
              if (u < hi) {
                VecG b = brow[u - u0];
                vec_fma(b, w, pv[q]);
                brow[u - u0] = b;
              }
            }
            row_unlock(row_locks + row);
          }
        } else {
          // spread: band_m[r][u] += wv[r] * P_m[u]; each profile read once
          // into registers (and cleared), one shared atomic per cell and row
#pragma unroll
          for (int m = 0; m < G; ++m) {
            float pv[CH];
            float *pm = prof + m * U;
#pragma unroll
            for (int q = 0; q < CH; ++q) {
              const int u = lo + lane + 32 * q;
              pv[q] = 0.f;
              if (u < hi) {
                pv[q] = pm[u - u0];
                pm[u - u0] = 0.f;
              }
            }
            float *bm = bands + (m * R + (rb - v0)) * U;
            for (int r = 0; r < nr; ++r) {
              const float w = wv[r];
              float *row = bm + r * U;
#pragma unroll
              for (int q = 0; q < CH; ++q) {
                const int u = lo + lane + 32 * q;
                if (u < hi) atomicAdd(row + (u - u0), w * pv[q]);
              }
            }
          }
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  const int nrow = v1 - v0, ncell = u1 - u0;
#pragma unroll
  for (int m = 0; m < G; ++m) {
    float *out = A.sino + (long)s_mem[m] * A.sino_view_stride;
    for (int t = threadIdx.x; t < nrow * ncell; t += blockDim.x) {
      const int r = t / ncell, u = t - r * ncell;
      out[(long)(v0 + r) * nu + u0 + u] += IL ? bands[(r * U + u) * G + m] : bands[(m * R + r) * U + u];
    }
  }
}

// ---------------------------------------------------------------------------
// Transpose over column orbits
// ---------------------------------------------------------------------------
// Orbit representative r -> column (i0, j0) of the fundamental domain:
// G = 4: the quadrant i, j < n/2; G = 2: rows j < ny/2 (ny even) or columns
// i < nx/2; G = 1: every column.
template <int G>
__device__ __forceinline__ void orbit_rep(int r, int nx, int ny, int &i0, int &j0)
{
  if constexpr (G == 4) {
    const int h = nx >> 1;
    i0 = r % h;
    j0 = r / h;
  } else if constexpr (G == 2) {
    if ((ny & 1) == 0) {
      i0 = r % nx;
      j0 = r / nx;
    } else {
      const int h = nx >> 1;
      i0 = r % h;
      j0 = r / h;
    }
  } else {
    i0 = r % nx;
    j0 = r / nx;
  }
}

template <int GEOM, int G, int KP>
__global__ void __launch_bounds__(256, 2)
k_back3d_group(const GroupBackLaunch A)
{
  extern __shared__ __align__(16) float sm[];
  const Params3D &P = A.P;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nz = P.nz, nx = P.nx, ny = P.ny;
  const int orbit = blockIdx.x * nwarps + warp;
  if (orbit >= A.norbits) return;
  using VecG = typename VecOf<G>::T;
  // v-collapsed member profiles, interleaved: cell u's G member values at
  // Q[u] (this warp's nu cells)
  VecG *Q = reinterpret_cast<VecG *>(sm) + warp * nu;
  int i0, j0;
  orbit_rep<G>(orbit, nx, ny, i0, j0);
  int oi[G], oj[G];
#pragma unroll
  for (int p = 0; p < G; ++p) turn_col(i0, j0, member_turn<G>(p), nx, ny, oi[p], oj[p]);
  const int kbase = blockIdx.y * (64 * KP);
  float2 acc[G][KP], cmp[G][KP];
#pragma unroll
  for (int q = 0; q < G; ++q)
#pragma unroll
    for (int p = 0; p < KP; ++p) {
      acc[q][p] = f2(0.f);
      cmp[q][p] = f2(0.f);
    }
  constexpr int GPB = 32 / G;  // groups whose columns one batch of lanes evaluates
  for (int gb = A.g_lo; gb < A.g_hi; gb += GPB) {
    // lane L: group gb + L / G, orbit member L % G
    ColGeo<MODEL_CUBIC> mine;
    {
      const int gg = gb + lane / G, p = lane % G;
      int pi = i0, pj = j0;
#pragma unroll
      for (int q = 0; q < G; ++q)
        if (q == p) {
          pi = oi[q];
          pj = oj[q];
        }
      if (gg < A.g_hi) {
        column_geo<GEOM, MODEL_CUBIC>(P, A.views[A.groups[4 * gg]], pi, pj, 0, mine);
        if (mine.bad) atomicOr(A.err, TRTT_ERR_SOURCE_PLANE);
      } else {
        mine.vax.n = 0;
        mine.bad = 1;
      }
    }
    const int ng = min(GPB, A.g_hi - gb);
    for (int s = 0; s < ng; ++s) {
      const int gg = gb + s;
      const View3D &V = A.views[A.groups[4 * gg]];
      const float *img[G];
#pragma unroll
      for (int m = 0; m < G; ++m) img[m] = A.sino + (long)A.groups[4 * gg + m] * A.sino_view_stride;
#pragma unroll
      for (int p = 0; p < G; ++p) {
        const int src = s * G + p;
        const int nvx = __shfl_sync(FULLM, mine.vax.n, src);
        const int bd = __shfl_sync(FULLM, mine.bad, src);
        if (bd || nvx <= 0) continue;
        const ColGeo<MODEL_CUBIC> cc = shfl_colc(mine, src);
        UPair up[KP];
        int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
        for (int kp = 0; kp < KP; ++kp) {
          const int k0 = kbase + lane + 64 * kp, k1 = k0 + 32;
          voxel_u_pair<GEOM>(P, V, cc, k0, k1, up[kp]);
          if (k0 >= nz) up[kp].n0 = 0;
          if (k1 >= nz) up[kp].n1 = 0;
          if (up[kp].n0 > 0) {
            lo = min(lo, up[kp].lo0);
            hi = max(hi, up[kp].lo0 + up[kp].n0);
          }
          if (up[kp].n1 > 0) {
            lo = min(lo, up[kp].lo1);
            hi = max(hi, up[kp].lo1 + up[kp].n1);
          }
        }
        lo = __reduce_min_sync(FULLM, lo);
        hi = __reduce_max_sync(FULLM, hi);
        if (lo >= hi) continue;
        // v-collapsed profiles of the member views over cells [lo, hi)
        const int npv = cc.vax.n;
        if (A.vec4) {
          // 16-byte loads of four cells and packed FMAs over the aligned
          // cover [lo & ~3, hi rounded up to 4) (nu % 4 == 0: rows and Q are
          // 16-byte aligned; the padding cells of Q are never read)
          constexpr int QV = G == 4 ? 1 : 2;  // float4 chunks per lane
          const int a0 = lo & ~3, a1 = (hi + 3) & ~3;
          for (int ub = a0; ub < a1; ub += 128 * QV) {
            float4 q[G][QV];
#pragma unroll
            for (int m = 0; m < G; ++m)
#pragma unroll
              for (int c = 0; c < QV; ++c) q[m][c] = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int m0 = 0; m0 < npv; m0 += 32) {
              const int mn = min(32, npv - m0);
              const float wl = (lane < mn) ? axis_weight<MODEL_CUBIC>(cc.vax, m0 + lane, P) : 0.f;
              for (int rr = 0; rr < mn; ++rr) {
                const float2 w = f2(__shfl_sync(FULLM, wl, rr));
                const long roff = (long)(cc.vax.lo + m0 + rr) * nu + ub + 4 * lane;
#pragma unroll
                for (int m = 0; m < G; ++m) {
                  const float4 *row = reinterpret_cast<const float4 *>(img[m] + roff);
#pragma unroll
                  for (int c = 0; c < QV; ++c) {
                    if (ub + 4 * lane + 128 * c < a1) {
                      const float4 y = __ldg(row + 32 * c);
                      const float2 lo2 = fma2(w, make_float2(y.x, y.y), make_float2(q[m][c].x, q[m][c].y));
                      const float2 hi2 = fma2(w, make_float2(y.z, y.w), make_float2(q[m][c].z, q[m][c].w));
                      q[m][c] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
                    }
                  }
                }
              }
            }
#pragma unroll
            for (int c = 0; c < QV; ++c) {
              const int u = ub + 4 * lane + 128 * c;
              if (u < a1) {
                float v[4][G];
#pragma unroll
                for (int m = 0; m < G; ++m) {
                  v[0][m] = comp<0>(q[m][c]);
                  v[1][m] = comp<1>(q[m][c]);
                  v[2][m] = comp<2>(q[m][c]);
                  v[3][m] = comp<3>(q[m][c]);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) pack(Q[u + j], v[j]);
              }
            }
          }
        } else {
        constexpr int QC = G == 4 ? 4 : 8;
        for (int ub = lo; ub < hi; ub += 32 * QC) {
          float q[G][QC];
#pragma unroll
          for (int m = 0; m < G; ++m)
#pragma unroll
            for (int c = 0; c < QC; ++c) q[m][c] = 0.f;
          for (int m0 = 0; m0 < npv; m0 += 32) {
            const int mn = min(32, npv - m0);
            const float wl = (lane < mn) ? axis_weight<MODEL_CUBIC>(cc.vax, m0 + lane, P) : 0.f;
            for (int rr = 0; rr < mn; ++rr) {
              const float w = __shfl_sync(FULLM, wl, rr);
              const long roff = (long)(cc.vax.lo + m0 + rr) * nu + ub + lane;
#pragma unroll
              for (int m = 0; m < G; ++m) {
                const float *row = img[m] + roff;
                float a[QC];
#pragma unroll
                for (int c = 0; c < QC; ++c) a[c] = (ub + lane + 32 * c < hi) ? __ldg(row + 32 * c) : 0.f;
#pragma unroll
                for (int c = 0; c < QC; ++c) q[m][c] = fmaf(w, a[c], q[m][c]);
              }
            }
          }
#pragma unroll
          for (int c = 0; c < QC; ++c)
            if (ub + lane + 32 * c < hi) {
              float v[G];
#pragma unroll
              for (int m = 0; m < G; ++m) v[m] = q[m][c];
              pack(Q[ub + lane + 32 * c], v);
            }
        }
        }
        __syncwarp();
        // per-voxel gathers, two voxels per instruction; member m's sum goes
        // to orbit column (p - m) mod G
#pragma unroll
        for (int kp = 0; kp < KP; ++kp) {
          const int L = max(up[kp].n0, up[kp].n1);
          if (L <= 0) continue;
          float2 Fp = first_edge_prim2(up[kp]);
          float2 S[G];
#pragma unroll
          for (int m = 0; m < G; ++m) S[m] = f2(0.f);
          float2 lf = f2(1.0f);
          const VecG *q0 = Q + up[kp].lo0;
          const VecG *q1 = Q + up[kp].lo1;
          for (int l = 0; l < L; ++l) {
            const float2 F = cubic_prim2(fma2(lf, up[kp].inc, up[kp].start));
            const float2 w = add2(F, make_float2(-Fp.x, -Fp.y));
            const VecG a0 = (l < up[kp].n0) ? q0[l] : VecG{};
            const VecG a1 = (l < up[kp].n1) ? q1[l] : VecG{};
            gather_fma<G>(S, w, a0, a1);
            Fp = F;
            lf = add2(lf, f2(1.0f));
          }
#pragma unroll
          for (int m = 0; m < G; ++m) {
            const int qo = (p - m + G) % G;
            const float2 term = mul2(up[kp].rho, S[m]);
            const float2 y = add2(term, make_float2(-cmp[qo][kp].x, -cmp[qo][kp].y));
            const float2 t = add2(acc[qo][kp], y);
            cmp[qo][kp] = add2(add2(t, make_float2(-acc[qo][kp].x, -acc[qo][kp].y)),
                               make_float2(-y.x, -y.y));
            acc[qo][kp] = t;
          }
        }
        __syncwarp();
      }
    }
  }
#pragma unroll
  for (int q = 0; q < G; ++q) {
    float *dst = A.vol + ((long)oj[q] * nx + oi[q]) * nz;
#pragma unroll
    for (int kp = 0; kp < KP; ++kp) {
      const int k0 = kbase + lane + 64 * kp, k1 = k0 + 32;
      if (k0 < nz) dst[k0] += acc[q][kp].x - cmp[q][kp].x;
      if (k1 < nz) dst[k1] += acc[q][kp].y - cmp[q][kp].y;
    }
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
namespace {

template <int GEOM, int G>
cudaError_t fwd_group(const GroupFwdLaunch &L, cudaStream_t st)
{
  if (L.ngroups <= 0) return cudaSuccess;
  const int nbands = (L.P.nv + L.band_rows - 1) / L.band_rows;
  dim3 grid(nbands * L.usplit, L.ngroups);
  const size_t smem = group_fwd_smem(G, L.band_rows, L.utile, L.warps);
  // register budget: 128 per thread (one 16-warp CTA per SM) or 64 (two);
  // groups of 1 and 2 views always fit two CTAs
  auto kern = (G == 4 && L.minb == 1)
                  ? (L.interleave ? k_fwd3d_group<GEOM, G, true, 1> : k_fwd3d_group<GEOM, G, false, 1>)
                  : (L.interleave ? k_fwd3d_group<GEOM, G, true, 2> : k_fwd3d_group<GEOM, G, false, 2>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, L.warps * 32, smem, st>>>(L);
  return cudaGetLastError();
}

template <int GEOM, int G>
cudaError_t back_group(const GroupBackLaunch &L, cudaStream_t st)
{
  if (L.g_hi <= L.g_lo || L.norbits <= 0) return cudaSuccess;
  constexpr int KP = 2;  // 2 voxel pairs per lane: 128 voxels of each orbit column per warp
  const int warps = 8;
  dim3 grid((L.norbits + warps - 1) / warps, (L.P.nz + 64 * KP - 1) / (64 * KP));
  const size_t smem = sizeof(float) * (size_t)warps * G * L.P.nu;
  auto kern = k_back3d_group<GEOM, G, KP>;
  // L.vec4 set by the caller: nu % 4 == 0 and 16-byte aligned images
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, warps * 32, smem, st>>>(L);
  return cudaGetLastError();
}

}  // namespace

size_t group_fwd_smem(int G, int band_rows, int utile, int warps)
{
  // bands, one profile and one row-weight list per warp, one lock per row
  return sizeof(float) * ((size_t)G * band_rows * utile + (size_t)warps * G * utile +
                          (size_t)warps * band_rows + (size_t)band_rows);
}

int group_fwd_warps(int G, int band_rows, int utile, int minb)
{
  // quads at one CTA per SM: 22 warps (up to 93 registers each) where the
  // bands and 22 profiles fit in shared memory, else 16
  if (G == 4 && minb == 1 && group_fwd_smem(4, band_rows, utile, 22) + 1024 <= 227u * 1024u) return 22;
  return 16;
}

int group_orbits(int G, int nx, int ny)
{
  if (G == 4) return (nx / 2) * (ny / 2);
  if (G == 2) return nx * ny / 2;
  return nx * ny;
}

cudaError_t launch_fwd3d_group(const GroupFwdLaunch &L, int G, cudaStream_t st)
{
  const bool cone = L.P.geom == GEOM_CONE;
  if (G == 4) return cone ? fwd_group<GEOM_CONE, 4>(L, st) : fwd_group<GEOM_PARALLEL, 4>(L, st);
  if (G == 2) return cone ? fwd_group<GEOM_CONE, 2>(L, st) : fwd_group<GEOM_PARALLEL, 2>(L, st);
  return cone ? fwd_group<GEOM_CONE, 1>(L, st) : fwd_group<GEOM_PARALLEL, 1>(L, st);
}

cudaError_t launch_back3d_group(const GroupBackLaunch &L, int G, cudaStream_t st)
{
  const bool cone = L.P.geom == GEOM_CONE;
  if (G == 4) return cone ? back_group<GEOM_CONE, 4>(L, st) : back_group<GEOM_PARALLEL, 4>(L, st);
  if (G == 2) return cone ? back_group<GEOM_CONE, 2>(L, st) : back_group<GEOM_PARALLEL, 2>(L, st);
  return cone ? back_group<GEOM_CONE, 1>(L, st) : back_group<GEOM_PARALLEL, 1>(L, st);
}

}  // namespace trtt
