// geom3d.cuh -- per-column and per-voxel geometry of the 3D B-spline
// projectors (parallel beam: plugin/trtt_3D_projectors.c:959-1075; cone
// beam: plugin/trtt_3D_projectors.c:1179-1338 and
// plugin/trtt_3D_projectors_cubic.c:623-778).
//
// Volumes are processed as voxel columns along k (the rotation axis).  For
// a circular orbit (xos a rotation about z, xsd a translation) the
// transaxial position vc, the magnification and the v-footprint of voxel
// (i,j,k) do not depend on k ("factorised" views, detected exactly on the
// host); the column state below is then computed once per column and view.
// For any other geometry it is recomputed per voxel (ColGeo at that k).
#pragma once

#include "trtt_device.cuh"

namespace trtt {

// Footprint axis in the representation of the model.
template <int MODEL> struct AxisOf { using type = AxisCubic; };
template <> struct AxisOf<MODEL_TABLE> { using type = AxisTable; };

// Transaxial (v) footprint of a column plus what the per-voxel u-footprint
// needs.
template <int MODEL>
struct ColGeo {
  typename AxisOf<MODEL>::type vax;
  int bad;          // voxel in the source plane (wk == 0): reference failure
  // cone beam
  double q;         // -a4/den
  double magn;      // -a4/wk
  double delta_v;
  double vca8sqr;
  double nyj, nxi;  // exact partial products of num_u (table mode)
  double A, B;      // closed-form mode: uc(k) = A + B k
  float h_u0m;      // h_u0 * magn
  float rho0c;      // rho0_init * magn^2 * delta_v (closed-form mode)
  float inv_den;    // 1 / (a4^2 + vca8^2)
};

// Edge value of the primitive along an axis.
template <int MODEL>
__device__ __forceinline__ float axis_weight(const typename AxisOf<MODEL>::type &ax,
                                             int l, const Params3D &P)
{
  if constexpr (MODEL == MODEL_TABLE) {
    double p0 = edge_table(ax, l, P.cum, P.last);
    double p1 = edge_table(ax, l + 1, P.cum, P.last);
    return (float)(p1 - p0);
  } else {
    return edge_cubic(ax, l + 1) - edge_cubic(ax, l);
  }
}

// Build an axis from its centre c, scale h, 1/h, half support hs, cell
// count n and clamp limit right_max.
template <int MODEL>
__device__ __forceinline__ void make_axis(typename AxisOf<MODEL>::type &ax,
                                          double c, double h, double scl,
                                          double hs, int n, int right_max,
                                          const Params3D &P)
{
  int lo = clamp_left_cell(dsub(c, hs), n);
  int hi = clamp_right_cell(dadd(c, hs), right_max);
  ax.lo = lo;
  ax.n = hi - lo;  // may be <= 0: empty footprint
  if constexpr (MODEL == MODEL_TABLE) {
    // ((left - c) - h*coord0) * (scl/step)   (plugin/trtt_3D_projectors.c:265-275)
    double s = ddiv(scl, P.step);
    ax.start = dmul(dsub(dsub((double)lo, c), dmul(h, P.coord0)), s);
    ax.inc = s;
  } else {
    // (left - c) * scl   (plugin/trtt_3D_projectors_cubic.c:253-254)
    ax.start = (float)dmul(dsub((double)lo, c), scl);
    ax.inc = (float)scl;
  }
}

// Closed-form (cubic) u axis from an FP64 centre and FP32 scales.
__device__ __forceinline__ void make_axis_fast(AxisCubic &ax, double c, float h,
                                               float scl, float hs, int n)
{
  int lo = clamp_left_cell(c - (double)hs, n);
  int hi = clamp_right_cell(c + (double)hs, n - 1);
  ax.lo = lo;
  ax.n = hi - lo;
  ax.start = (float)((double)lo - c) * scl;
  ax.inc = scl;
  (void)h;
}

// Column state of (i,j) evaluated at slice k (k = 0 for factorised views).
template <int GEOM, int MODEL>
__device__ __forceinline__ void column_geo(const Params3D &P, const View3D &V,
                                           int i, int j, int k,
                                           ColGeo<MODEL> &c)
{
  const double di = (double)i, dj = (double)j, dk = (double)k;
  c.bad = 0;
  if constexpr (GEOM == GEOM_CONE) {
    // wk, num_v, den in the reference's summation order (:1234-1251)
    double wk = dadd(dadd(dadd(dmul(V.o3, dk), V.o4), dmul(V.o2, dj)), dmul(V.o1, di));
    double num_v = dadd(dadd(dadd(dmul(V.nv_z, dk), V.nv_c), dmul(V.nv_y, dj)), dmul(V.nv_x, di));
    double den = dadd(dadd(dadd(dmul(V.d_z, dk), V.d_c), dmul(V.d_y, dj)), dmul(V.d_x, di));
    double q = ddiv(V.a4m, den);
    double vc = dadd(dmul(q, num_v), V.b3);
    c.q = q;
    if (wk == 0.0) {
      c.bad = 1;
      c.vax.lo = 0;
      c.vax.n = 0;
      return;
    }
    if (!isfinite(vc)) {  // den == 0: zero-weight footprint in the reference
      c.vax.lo = 0;
      c.vax.n = 0;
      return;
    }
    double vca8 = dmul(dsub(vc, V.a8), P.v_scl);
    double vca8sqr = dmul(vca8, vca8);
    double magn = ddiv(V.a4m, wk);
    double delta_v = dsqrt(dadd(1.0, ddiv(vca8sqr, V.a4sqr)));
    double h_v = dmul(dmul(P.h_v0, magn), delta_v);
    double scl_v = ddiv(1.0, h_v);
    make_axis<MODEL>(c.vax, vc, h_v, scl_v, dmul(P.hs0, h_v), P.nv, P.nv - 1, P);
    c.magn = magn;
    c.delta_v = delta_v;
    c.vca8sqr = vca8sqr;
    c.nyj = dmul(V.nu_y, dj);
    c.nxi = dmul(V.nu_x, di);
    double num_u0 = dadd(dadd(V.nu_c, c.nyj), c.nxi);
    c.A = fma(q, num_u0, V.c3);
    c.B = q * V.nu_z;
    c.h_u0m = (float)(P.h_u0 * magn);
    c.rho0c = (float)(P.rho0_init * (magn * magn) * delta_v);
    c.inv_den = (float)(1.0 / (V.a4sqr + vca8sqr));
  } else {
    double vc = dadd(dadd(dadd(dmul(V.v_z, dk), V.v_c), dmul(V.v_y, dj)), dmul(V.v_x, di));
    if (!isfinite(vc)) {
      c.vax.lo = 0;
      c.vax.n = 0;
      return;
    }
    make_axis<MODEL>(c.vax, vc, V.p_h_v, V.p_scl_v, V.p_hs_v, P.nv, P.nv - 1, P);
    c.nyj = dmul(V.u_y, dj);
    c.nxi = dmul(V.u_x, di);
    c.A = dadd(dadd(V.u_c, c.nyj), c.nxi);
    c.B = V.u_z;
  }
}

// u footprint and weighting factor rho0 of voxel k of a column.  Returns
// false when the footprint is empty.
template <int GEOM, int MODEL>
__device__ __forceinline__ bool voxel_u(const Params3D &P, const View3D &V,
                                        const ColGeo<MODEL> &c, int k,
                                        typename AxisOf<MODEL>::type &ax,
                                        float &rho0)
{
  const double dk = (double)k;
  if constexpr (GEOM == GEOM_CONE) {
    if constexpr (MODEL == MODEL_TABLE) {
      // exact FP64 path, reference order (:1253-1280)
      double num_u = dadd(dadd(dadd(dmul(V.nu_z, dk), V.nu_c), c.nyj), c.nxi);
      double uc = dadd(dmul(c.q, num_u), V.c3);
      double uca12 = dmul(dsub(uc, V.a12), P.u_scl);
      double delta_u = dsqrt(dadd(1.0, ddiv(dmul(uca12, uca12), dadd(V.a4sqr, c.vca8sqr))));
      double r = dmul(dmul(dmul(P.rho0_init, dmul(c.magn, c.magn)), delta_u), c.delta_v);
      double h_u = dmul(dmul(P.h_u0, c.magn), delta_u);
      double scl_u = ddiv(1.0, h_u);
      make_axis<MODEL>(ax, uc, h_u, scl_u, dmul(P.hs0, h_u), P.nu, P.nu - 1, P);
      rho0 = (float)r;
    } else {
      double uc = fma(c.B, dk, c.A);
      float uca12 = (float)(uc - V.a12) * (float)P.u_scl;
      float du2 = fmaf(uca12 * uca12, c.inv_den, 1.0f);
      float delta_u = du2 * rsqrtf(du2);
      float h_u = c.h_u0m * delta_u;
      float scl_u = __frcp_rn(h_u);
      make_axis_fast(ax, uc, h_u, scl_u, (float)P.hs0 * h_u, P.nu);
      rho0 = c.rho0c * delta_u;
    }
  } else {
    if constexpr (MODEL == MODEL_TABLE) {
      double uc = dadd(dadd(dadd(dmul(V.u_z, dk), V.u_c), c.nyj), c.nxi);
      make_axis<MODEL>(ax, uc, V.p_h_u, V.p_scl_u, V.p_hs_u, P.nu, P.nu - 1, P);
    } else {
      double uc = fma(c.B, dk, c.A);
      make_axis_fast(ax, uc, (float)V.p_h_u, (float)V.p_scl_u, (float)V.p_hs_u, P.nu);
    }
    rho0 = (float)V.p_rho0;
  }
  return ax.n > 0 && isfinite(ax.start);
}

}  // namespace trtt
