// fast3d.cuh -- packed-FP32 (f32x2) evaluation of the closed-form cubic
// footprint for two voxels at a time (sm_100a FFMA2/FMUL2/FADD2).
//
// The direct and transpose kernels of the cubic model both call
// voxel_u_pair() and cubic_prim2(), so the pair stays an exact adjoint.
#pragma once

#include <climits>

#include "geom3d.cuh"

namespace trtt {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Cubic B-spline primitive at two abscissae.  With t = |x| the tail mass
// beyond t is g(t) = ((2-t)_+^4 - 4 (1-t)_+^4) / 24 (truncated-power form of
// the centred cubic B-spline), and P(x) = 1/2 + sign(x) (1/2 - g(|x|)).
// Expanding gives the four quartics of
// plugin/trtt_3D_projectors_cubic.c:117-138; agreement is to FP32 rounding.
__device__ __forceinline__ float2 cubic_prim2(float2 x)
{
  const float2 t = make_float2(fabsf(x.x), fabsf(x.y));
  float2 a = fma2(t, f2(-1.0f), f2(2.0f));
  float2 b = fma2(t, f2(-1.0f), f2(1.0f));
  a = make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f));
  b = make_float2(fmaxf(b.x, 0.0f), fmaxf(b.y, 0.0f));
  const float2 a2 = mul2(a, a), b2 = mul2(b, b);
  const float2 a4 = mul2(a2, a2), b4 = mul2(b2, b2);
  const float2 g = fma2(a4, f2(0.0416666666666667f), mul2(b4, f2(-0.1666666666666667f)));
  const float2 h = fma2(g, f2(-1.0f), f2(0.5f));  // 1/2 - g
  return add2(make_float2(copysignf(h.x, x.x), copysignf(h.y, x.y)), f2(0.5f));
}

// u-footprints of two voxels of one column (closed-form model): cells
// [lo, lo+n) and edge abscissae start + l*inc, weighting factors rho.
struct UPair {
  int lo0, n0, lo1, n1;
  float2 start, inc, rho;
};

template <int GEOM>
__device__ __forceinline__ void voxel_u_pair(const Params3D &P, const View3D &V,
                                             const ColGeo<MODEL_CUBIC> &c, int k0, int k1,
                                             UPair &up)
{
  const double uc0 = fma(c.B, (double)k0, c.A);
  const double uc1 = fma(c.B, (double)k1, c.A);
  float2 scl, hs;
  if constexpr (GEOM == GEOM_CONE) {
    const float2 d = make_float2((float)(uc0 - V.a12), (float)(uc1 - V.a12));
    const float2 uca = mul2(d, f2((float)P.u_scl));
    const float2 du2 = fma2(mul2(uca, uca), f2(c.inv_den), f2(1.0f));
    const float2 dlt = mul2(du2, make_float2(rsqrtf(du2.x), rsqrtf(du2.y)));
    const float2 h = mul2(dlt, f2(c.h_u0m));
    scl = make_float2(__fdividef(1.0f, h.x), __fdividef(1.0f, h.y));  // 2 ulp, h in (0, 2^126)
    hs = mul2(h, f2((float)P.hs0));
    up.rho = mul2(dlt, f2(c.rho0c));
  } else {
    scl = f2((float)V.p_scl_u);
    hs = f2((float)V.p_hs_u);
    up.rho = f2((float)V.p_rho0);
  }
  const int n = P.nu;
  up.lo0 = clamp_left_cell(uc0 - (double)hs.x, n);
  up.n0 = clamp_right_cell(uc0 + (double)hs.x, n - 1) - up.lo0;
  up.lo1 = clamp_left_cell(uc1 - (double)hs.y, n);
  up.n1 = clamp_right_cell(uc1 + (double)hs.y, n - 1) - up.lo1;
  const float2 off = make_float2((float)((double)up.lo0 - uc0), (float)((double)up.lo1 - uc1));
  up.start = mul2(off, scl);
  up.inc = scl;
  if (!(isfinite(up.start.x) && isfinite(scl.x))) up.n0 = 0;
  if (!(isfinite(up.start.y) && isfinite(scl.y))) up.n1 = 0;
}

// Primitive at the first edge of both voxels of a pair.  A cell range that
// was not clamped at cell 0 starts at floor(uc - hs), at or left of the
// support start, where the primitive is 0 (to within FP32 rounding of the
// edge abscissa, below 1e-24); only ranges clamped at the detector's first
// cell need the evaluation.  Used by the direct and transpose kernels alike.
__device__ __forceinline__ float2 first_edge_prim2(const UPair &up)
{
  if (up.lo0 > 0 && up.lo1 > 0) return f2(0.0f);
  return cubic_prim2(up.start);
}

// Column helpers shared by the direct kernels ----------------------------

static constexpr unsigned FULLM = 0xffffffffu;

__device__ __forceinline__ ColGeo<MODEL_CUBIC> shfl_colc(const ColGeo<MODEL_CUBIC> &c, int src)
{
  ColGeo<MODEL_CUBIC> r;
  r.vax.lo = __shfl_sync(FULLM, c.vax.lo, src);
  r.vax.n = __shfl_sync(FULLM, c.vax.n, src);
  r.vax.start = __shfl_sync(FULLM, c.vax.start, src);
  r.vax.inc = __shfl_sync(FULLM, c.vax.inc, src);
  r.bad = 0;
  r.A = __shfl_sync(FULLM, c.A, src);
  r.B = __shfl_sync(FULLM, c.B, src);
  r.h_u0m = __shfl_sync(FULLM, c.h_u0m, src);
  r.rho0c = __shfl_sync(FULLM, c.rho0c, src);
  r.inv_den = __shfl_sync(FULLM, c.inv_den, src);
  return r;
}

__device__ __forceinline__ float vox_val(const float *__restrict__ vol, long gate_stride,
                                         const View3D &V, long idx)
{
  float x = __ldg(vol + (long)V.g0 * gate_stride + idx);
  if (V.w1 != 0.0f) return fmaf(V.w0, x, V.w1 * __ldg(vol + (long)V.g1 * gate_stride + idx));
  return V.w0 == 1.0f ? x : V.w0 * x;
}

// Profile of one column: prof[u] += sum_k rho_k x_k (F(e_{u+1,k}) - F(e_{u,k}))
// (shared-memory atomics), returns the warp-uniform cell range [lo, hi).
template <int GEOM>
__device__ __forceinline__ void column_profile(const Params3D &P, const View3D &V, const float *__restrict__ vol,
                                               long gate_stride, const ColGeo<MODEL_CUBIC> &cc, int col,
                                               float *prof, int lane, int &lo_out, int &hi_out)
{
  const int nz = P.nz;
  int lo = INT_MAX, hi = INT_MIN;
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
  lo_out = __reduce_min_sync(FULLM, lo);
  hi_out = __reduce_max_sync(FULLM, hi);
}

}  // namespace trtt
