// host3d.h -- host-side derivation of the 3D projector parameters shared by
// the C ABI translation units (plan, drop-in and allocation-free entry
// points).
#pragma once

#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "trtt_b200.h"

namespace trtt {

// Per-view constants of the 3D projectors, derived in FP64 with the operand
// order of the reference so that the device sees the reference's values
// (cone beam plugin/trtt_3D_projectors.c:1186-1230, parallel beam
// plugin/trtt_3D_projectors.c:963-1004; identical in the _cubic file).
inline void make_view3d(const Params3D &P, const double *xos, const double *xsd, View3D &V)
{
  std::memset(&V, 0, sizeof(V));
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o1 = xos[0], o2 = xos[1], o3 = xos[2], o4 = xos[3];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  const double a1inv = -1.0 * (1.0 / a1);
  const double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  const double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  const double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  V.o1 = o1; V.o2 = o2; V.o3 = o3; V.o4 = o4;
  V.nv_x = b1 * o5 + b2 * o9;  V.nu_x = c1 * o5 + c2 * o9;
  V.nv_y = b1 * o6 + b2 * o10; V.nu_y = c1 * o6 + c2 * o10;
  V.nv_z = b1 * o7 + b2 * o11; V.nu_z = c1 * o7 + c2 * o11;
  V.nv_c = b1 * o8 + b2 * o12; V.nu_c = c1 * o8 + c2 * o12;
  V.d_x = a1 * o1 + a2 * o5 + a3 * o9;
  V.d_y = a1 * o2 + a2 * o6 + a3 * o10;
  V.d_z = a1 * o3 + a2 * o7 + a3 * o11;
  V.d_c = a1 * o4 + a2 * o8 + a3 * o12;
  V.a4sqr = a4 * a4;
  V.a4m = -1.0 * a4;
  V.a8 = a8;
  V.a12 = a12;
  V.b3 = b3;
  V.c3 = c3;
  // parallel beam
  V.v_x = b1 * o5 + b2 * o9;  V.u_x = c1 * o5 + c2 * o9;
  V.v_y = b1 * o6 + b2 * o10; V.u_y = c1 * o6 + c2 * o10;
  V.v_z = b1 * o7 + b2 * o11; V.u_z = c1 * o7 + c2 * o11;
  V.v_c = b1 * o8 + b2 * o12 + b3; V.u_c = c1 * o8 + c2 * o12 + c3;
  const double a1sqr = a1 * a1;
  const double a5sqr = P.v_scl * P.v_scl * a5 * a5;
  const double a9sqr = P.u_scl * P.u_scl * a9 * a9;
  const double delta_u = std::sqrt(1.0 + (a9sqr / (a1sqr + a5sqr)));
  const double delta_v = std::sqrt(1.0 + (a5sqr / a1sqr));
  V.p_rho0 = P.s_scl * P.s_scl * P.s_scl * delta_u * delta_v;
  V.p_h_u = P.s_scl / P.u_scl;
  V.p_h_v = P.s_scl / P.v_scl;
  V.p_scl_u = 1.0 / V.p_h_u;
  V.p_scl_v = 1.0 / V.p_h_v;
  V.p_hs_u = P.hs0 * V.p_h_u;
  V.p_hs_v = P.hs0 * V.p_h_v;
  V.p_sclt_u = V.p_scl_u / P.step;
  V.p_sclt_v = V.p_scl_v / P.step;
  V.g0 = 0;
  V.g1 = 0;
  V.w0 = 1.0f;
  V.w1 = 0.0f;
  if (P.geom == GEOM_CONE)
    V.factorized = (V.o3 == 0.0 && V.d_z == 0.0 && V.nv_z == 0.0) ? 1 : 0;
  else
    V.factorized = (V.v_z == 0.0) ? 1 : 0;
}

inline Params3D make_params(int geom, long nx, long ny, long nz, double s_scl, int s_deg,
                     const double *cum_dev, long size, double step,
                     double coord0, long nu, long nv, double u_scl, double v_scl)
{
  Params3D P;
  std::memset(&P, 0, sizeof(P));
  P.geom = geom;
  P.model = cum_dev ? MODEL_TABLE : MODEL_CUBIC;
  P.nx = (int)nx; P.ny = (int)ny; P.nz = (int)nz;
  P.nu = (int)nu; P.nv = (int)nv;
  P.nt = 1;
  P.s_scl = s_scl;
  P.u_scl = u_scl;
  P.v_scl = v_scl;
  P.rho0_init = s_scl * s_scl * s_scl;
  P.h_u0 = s_scl / u_scl;
  P.h_v0 = s_scl / v_scl;
  P.hs0 = 0.5 * (s_deg + 1);
  P.cum = cum_dev;
  P.size = (int)size;
  P.last = (double)(size - 1);
  P.step = cum_dev ? step : 1.0;
  P.coord0 = coord0;
  return P;
}

// Size limits shared by every 3D entry point that takes device arrays:
// dimensions in [1, 2^30) (int indices in the kernels), one volume slice
// below 2^31 voxels and the whole volume below 2^40.  Returns nullptr when
// the sizes are accepted, else the reason.
inline const char *check_sizes3d(long nx, long ny, long nz, long nu, long nv, long nviews)
{
  auto ok = [](long n) { return n >= 1 && n < (1L << 30); };
  if (!ok(nx) || !ok(ny) || !ok(nz) || !ok(nu) || !ok(nv) || !ok(nviews))
    return "sizes must be in [1, 2^30)";
  if (nx * ny >= (1L << 31) || nx * ny * nz >= (1L << 40)) return "volume too large";
  return nullptr;
}

// ---------------------------------------------------------------------------
// Orbit symmetry of a scan's views.  R(i, j) = (n-1-j, i) is the quarter turn
// of a square grid about the z axis, R^2(i, j) = (nx-1-i, ny-1-j) the half
// turn of any grid.  View b is the m-turn image of view a when it sees voxel
// (i, j, k) where view a sees voxel (R^m(i, j), k): its xos rows (p, q, r, s)
// acting as p i + q j + r k + s equal those of view a with the substitution
// applied, and its xsd equals view a's.  The footprints of view b's voxel
// column c are then view a's footprints of column R^m(c), so a group of
// views needs the footprint arithmetic of its first view only.
// ---------------------------------------------------------------------------
inline void turn_xos(const double *x, int m, long nx, long ny, double *out)
{
  for (int r = 0; r < 3; ++r) {
    const double a = x[4 * r], b = x[4 * r + 1], c = x[4 * r + 2], d = x[4 * r + 3];
    double *o = out + 4 * r;
    o[2] = c;
    if (m == 1) {
      o[0] = b; o[1] = -a; o[3] = d + a * (double)(nx - 1);
    } else if (m == 2) {
      o[0] = -a; o[1] = -b; o[3] = d + a * (double)(nx - 1) + b * (double)(ny - 1);
    } else if (m == 3) {
      o[0] = -b; o[1] = a; o[3] = d + b * (double)(ny - 1);
    } else {
      o[0] = a; o[1] = b; o[3] = d;
    }
  }
}

// Rows of two 3x4 matrices equal within tol relative to the row's magnitude.
inline bool coefs_match(const double *p, const double *q, double tol)
{
  for (int r = 0; r < 3; ++r) {
    double s = 0.0;
    for (int c = 0; c < 4; ++c) s = std::fmax(s, std::fmax(std::fabs(p[4 * r + c]), std::fabs(q[4 * r + c])));
    for (int c = 0; c < 4; ++c)
      if (!(std::fabs(p[4 * r + c] - q[4 * r + c]) <= tol * s)) return false;
  }
  return true;
}

// Greedy grouping in view order: {a, b1, b2, b3} (quarter turns, square grid
// of even side), else {a, b2} (half turn, nx or ny even), else {a}.  Each
// group is written as four view indices (unused slots -1) into the list of
// its size: groups[0] singles, groups[1] pairs, groups[2] quads.
inline void find_view_groups(long nx, long ny, long nviews, const double *xos, const double *xsd,
                             std::vector<int> groups[3], double tol = 1e-10)
{
  std::vector<char> used(nviews, 0);
  const bool quad_ok = nx == ny && nx % 2 == 0;
  const bool pair_ok = nx % 2 == 0 || ny % 2 == 0;
  auto find = [&](const double *coefs, const double *xd) -> long {
    for (long b = 0; b < nviews; ++b)
      if (!used[b] && coefs_match(xos + 12 * b, coefs, tol) && coefs_match(xsd + 12 * b, xd, tol))
        return b;
    return -1;
  };
  double t[12];
  for (long a = 0; a < nviews; ++a) {
    if (used[a]) continue;
    used[a] = 1;
    long mem[4] = {a, -1, -1, -1};
    int n = 1;
    if (quad_ok) {
      long b[3];
      for (int m = 1; m <= 3; ++m) {
        turn_xos(xos + 12 * a, m, nx, ny, t);
        b[m - 1] = find(t, xsd + 12 * a);
      }
      if (b[0] >= 0 && b[1] >= 0 && b[2] >= 0 && b[0] != b[1] && b[0] != b[2] && b[1] != b[2]) {
        mem[1] = b[0]; mem[2] = b[1]; mem[3] = b[2];
        n = 4;
      }
    }
    if (n == 1 && pair_ok) {
      turn_xos(xos + 12 * a, 2, nx, ny, t);
      const long b2 = find(t, xsd + 12 * a);
      if (b2 >= 0) {
        mem[1] = b2;
        n = 2;
      }
    }
    for (int m = 1; m < n; ++m) used[mem[m]] = 1;
    std::vector<int> &dst = groups[n == 4 ? 2 : n - 1];
    for (int m = 0; m < 4; ++m) dst.push_back((int)mem[m]);
  }
}

// Band shape of the direct kernel for a detector nu cells wide.
inline void choose_band(int nu, int nv, int &band_rows, int &warps)
{
  const long budget = 200 * 1024;
  warps = 16;
  while (warps > 2 && (long)warps * nu * 4 > budget / 3) warps /= 2;
  const long rest = budget - (long)warps * nu * 4;
  long rows = rest / ((long)nu * 4 + (long)warps * 4);
  if (rows > 32) rows = 32;  // two CTAs (2 x 16 warps) per SM at nu = 512
  if (rows > nv) rows = nv;
  band_rows = rows >= 2 ? (int)rows : 0;
}

inline int geom_code(int geometry)
{
  if (geometry == TRTT_B200_PARALLEL_BEAM) return GEOM_PARALLEL;
  if (geometry == TRTT_B200_CONE_BEAM || geometry == TRTT_B200_FAN_BEAM) return GEOM_CONE;
  return -1;
}

}  // namespace trtt
