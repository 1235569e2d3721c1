// trtt_device.cuh -- device-side footprint and geometry primitives shared by
// every projector kernel (direct and transpose use the same functions, so
// each pair is an adjoint pair up to FP32 summation rounding).
//
// Precision policy
//  * Table mode (trtt_PB2D/FB2D/PB3D/CB3D): the footprint is read from the
//    cumulative table at floor() of a continuous index of magnitude up to
//    size_footprint.  That index is computed in FP64 with the operation order
//    of the reference and no fused multiply-add (explicit __d*_rn
//    intrinsics), so the floor lands on the same table slot as the FP64
//    reference.
//  * Closed-form cubic mode: footprint centres and cell bounds are FP64
//    (positions of hundreds of cells need ~1e-7 absolute accuracy); scale
//    factors, B-spline primitives and weights are FP32.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "trtt_types.h"

namespace trtt {

// ---------------------------------------------------------------------------
// Exact FP64 arithmetic helpers (no contraction into FMA).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// ---------------------------------------------------------------------------
// Cubic B-spline primitive: integral of the centred cubic B-spline from
// -inf to x (plugin/trtt_3D_projectors_cubic.c:117-138).  FP32 form written
// around |x|: for t=|x| the tail mass beyond t is
//   (2-t)^4/24                          for 1 < t < 2
//   1/2 - t (2/3 - t^2 (1/3 - t/8))     for t <= 1
// and the primitive is the tail mass for x <= 0, one minus it for x > 0;
// expanding these gives the reference's four quartics.  The coefficients
// are the reference's decimal literals (plugin/trtt_3D_projectors_cubic.c:46-50)
// rounded to float.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float cubic_prim_f(float x)
{
  const float k24 = 0.0416666666666667f, k3 = 0.3333333333333333f;
  const float k23 = 0.6666666666666666f, k8 = 0.125f;
  float t = fabsf(x);
  float a = fmaxf(2.0f - t, 0.0f);
  float a2 = a * a;
  float outer = a2 * a2 * k24;
  float t2 = t * t;
  float inner = fmaf(-t, fmaf(-t2, fmaf(-t, k8, k3), k23), 0.5f);
  float g = (t > 1.0f) ? outer : inner;
  return (x <= 0.0f) ? g : 1.0f - g;
}

// FP64 form of the same primitive, operation order of the reference
// (used by the exact-arithmetic paths of the 2D cubic projectors).
__device__ __forceinline__ double cubic_prim_d(double x)
{
  const double K24 = 0.0416666666666667, K3 = 0.3333333333333333;
  const double K23 = 0.6666666666666666, K43 = 1.3333333333333333, K8 = 0.125;
  double x2 = dmul(x, x);
  double x3 = dmul(x2, x);
  double x4 = dmul(x, x3);
  if (x <= -2.0) return 0.0;
  if (x <= -1.0)
    return dadd(dadd(dadd(dadd(dmul(K24, x4), dmul(K3, x3)), x2), dmul(K43, x)), K23);
  if (x <= 0.0)
    return dadd(dadd(dsub(dmul(dmul(-1.0, K8), x4), dmul(K3, x3)), dmul(K23, x)), 0.5);
  if (x <= 1.0)
    return dadd(dadd(dsub(dmul(K8, x4), dmul(K3, x3)), dmul(K23, x)), 0.5);
  if (x < 2.0)
    return dadd(dadd(dsub(dadd(dmul(dmul(-1.0, K24), x4), dmul(K3, x3)), x2), dmul(K43, x)), K3);
  return 1.0;
}

// ---------------------------------------------------------------------------
// Table lookup slot floor(min(max(x,0), m-1))  (plugin/trtt_3D_projectors.c:288-297).
// fmax(NaN,0)=0 reproduces the reference's MAX macro on NaN.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int table_slot(double x, double last)
{
  double t = fmax(x, 0.0);
  t = fmin(t, last);
  return __double2int_rd(t);
}

// ---------------------------------------------------------------------------
// Detector-cell bounds with the reference's clamps
// (plugin/trtt_3D_projectors.c:1292-1307): left = clamp(floor(c-hs), 0, n-1),
// right = clamp(floor(c+hs)+1, 0, right_max+1).  right_max is n-1 except for
// the 2D closed-form cubic projectors (n-2).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int clamp_left_cell(double t, int n)
{
  int f = __double2int_rd(t);
  return min(max(f, 0), n - 1);
}
__device__ __forceinline__ int clamp_right_cell(double t, int right_max)
{
  int f = __double2int_rd(t);
  f = (f == INT32_MAX) ? f : f + 1;
  return min(max(f, 0), right_max + 1);
}

// ---------------------------------------------------------------------------
// One axis of a voxel footprint: cells [lo, lo+n) of a detector axis and the
// normalised coordinates of their edges.
// ---------------------------------------------------------------------------
struct AxisCubic {     // closed-form cubic: edge l at start + l*inc (FP32)
  int lo, n;
  float start, inc;
};
struct AxisTable {     // table: edge l at start + l*inc (FP64, exact)
  int lo, n;
  double start, inc;
};

// Primitive value at edge l.
__device__ __forceinline__ float edge_cubic(const AxisCubic &a, int l)
{
  return cubic_prim_f(fmaf((float)l, a.inc, a.start));
}
__device__ __forceinline__ double edge_table(const AxisTable &a, int l,
                                             const double *__restrict__ cum,
                                             double last)
{
  double x = (l == 0) ? a.start : dadd(a.start, dmul((double)l, a.inc));
  return __ldg(cum + table_slot(x, last));
}

// Kahan-compensated accumulation.
struct Kahan {
  float s, c;
  __device__ __forceinline__ Kahan() : s(0.f), c(0.f) {}
  __device__ __forceinline__ void add(float v)
  {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s - c; }
};

}  // namespace trtt
