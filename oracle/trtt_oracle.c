/*
 * trtt_oracle.c -- FP64 CPU restatement of the TRTT projector plugin.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker).  Nothing in the product
 * package calls this code; the B200 kernels are checked against it.
 *
 * Each routine restates the reference routine cited beside it, keeping the
 * operand order of every floating-point expression (and no fused
 * multiply-add: build with -ffp-contract=off) so that its output is
 * bit-identical to the reference plugin compiled from its own sources.  The
 * structure differs from the reference: one footprint-weight helper serves
 * every geometry, the 1D weights of a voxel are computed into a scratch row
 * allocated once per call instead of once per voxel, and the 2D/3D drivers
 * share their clamp and table-lookup helpers.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "trtt_oracle.h"

#define ORC_SUCCESS (0)
#define ORC_FAILURE (-1)

/* ------------------------------------------------------------------------ */
/* Footprint primitives                                                      */
/* ------------------------------------------------------------------------ */

/* Decimal literals used by the reference for the cubic B-spline primitive
 * (plugin/trtt_3D_projectors_cubic.c:46-50, identical in the 2D file). */
#define C24 0.0416666666666667
#define C3 0.3333333333333333
#define C23 0.6666666666666666
#define C43 1.3333333333333333
#define C8 0.125

/* Integral of the centred cubic B-spline from -inf to x
 * (plugin/trtt_3D_projectors_cubic.c:117-138, plugin/trtt_2D_projectors_cubic.c:73-94).
 * A NaN argument falls through every test and yields 1, as in the
 * reference. */
static double cubic_primitive(double x)
{
  double x2 = x * x;
  double x3 = x2 * x;
  if (x <= -2.0) return 0.0;
  if (x <= -1.0) return C24 * (x * x3) + C3 * x3 + x2 + C43 * x + C23;
  if (x <= 0.0) return (-1.0) * C8 * (x * x3) - C3 * x3 + C23 * x + 0.5;
  if (x <= 1.0) return C8 * (x * x3) - C3 * x3 + C23 * x + 0.5;
  if (x < 2.0) return (-1.0) * C24 * (x * x3) + C3 * x3 - x2 + C43 * x + C3;
  return 1.0;
}

/* Floor-indexed table lookup position: floor(min(max(x,0), m-1))
 * (plugin/trtt_3D_projectors.c:288-297, plugin/trtt_2D_projectors.c:106-111). */
static long table_slot(double x, long m)
{
  double t = (x >= 0) ? x : 0;
  double last = (double)(m - 1);
  t = (t <= last) ? t : last;
  return (long)floor(t);
}

/* Left / right detector bounds of a footprint centred at c with half
 * support hs, clamped as in plugin/trtt_3D_projectors.c:1292-1307.  The
 * right bound saturates at right_max+1 where right_max is n-1 except for the
 * 2D closed-form cubic projectors, which use n-2
 * (plugin/trtt_2D_projectors_cubic.c:254-258). */
static double clamp_left(double t, long n)
{
  if (t < 0.0) return 0.0;
  if (t >= 0.0 && t <= (n - 1)) return floor(t);
  return (double)(n - 1);
}
static double clamp_right(double t, long right_max)
{
  if (t < 0.0) return 0.0;
  if (t >= 0.0 && t <= right_max) return floor(t) + 1;
  return (double)(right_max + 1);
}

/* Footprint model shared by every B-spline projector. */
typedef struct {
  int table;              /* 0: closed-form cubic primitive; 1: table */
  const double *cum;      /* cumulative footprint table (table mode) */
  long m;                 /* table size */
} orc_model;

static double model_primitive(const orc_model *md, double x)
{
  return md->table ? md->cum[table_slot(x, md->m)] : cubic_primitive(x);
}

/* Weights of n consecutive detector cells whose lower edges sit at
 * normalised footprint coordinates start, start+inc, ...:
 *   w[l] = P(start + (l+1)*inc) - P(start + l*inc)
 * with P the model primitive, evaluated in the same sequence as the
 * reference loops (plugin/trtt_3D_projectors.c:293-306). */
static void cell_weights(const orc_model *md, double start, double inc, long n,
                         double *w)
{
  long l;
  double p0 = model_primitive(md, start);
  for (l = 0; l < n; ++l) {
    double x = start + (l + 1) * inc;
    double p1 = model_primitive(md, x);
    w[l] = p1 - p0;
    p0 = p1;
  }
}

/* ------------------------------------------------------------------------ */
/* 3D separable footprint burn (direct and transpose)                        */
/* ------------------------------------------------------------------------ */

/* One voxel of a 3D B-spline projector: weights along u and v, then either
 *   direct:    out[v,u]  += ((cv*cu)*vox)*rho0
 *   transpose: vox_acc   += ((rho0*cu)*cv)*pix[v,u]
 * (plugin/trtt_3D_projectors.c:231-329 and :628-730, cubic twin
 *  plugin/trtt_3D_projectors_cubic.c:231-307 and :410-491).
 * start_u/start_v and inc_u/inc_v are already in the model's normalised
 * coordinate (table index units or B-spline units). */
static void burn3d(const orc_model *md, int job, double *pix, double vox,
                   double *vox_acc, double ul, double ur, double vl, double vr,
                   long nu, double rho0, double start_u, double inc_u,
                   double start_v, double inc_v, double *wu)
{
  long l, m, npu, npv, base;
  double pv0;
  if (!(ul < ur && vl < vr)) return;
  npu = (long)(ur - ul);
  npv = (long)(vr - vl);
  base = (long)vl * nu + (long)ul;
  cell_weights(md, start_u, inc_u, npu, wu);
  pv0 = model_primitive(md, start_v);
  for (m = 0; m < npv; ++m) {
    double x = start_v + (m + 1) * inc_v;
    double pv1 = model_primitive(md, x);
    double cv = pv1 - pv0;
    long row = base + m * nu;
    if (job == 0) {
      for (l = 0; l < npu; ++l) pix[row + l] += cv * wu[l] * vox * rho0;
    } else {
      for (l = 0; l < npu; ++l) *vox_acc += rho0 * wu[l] * cv * pix[row + l];
    }
    pv0 = pv1;
  }
}

/* Normalised start coordinate and increment for the 3D drivers.
 * Table mode: ((left-c) - h*coord0) * (scl/step)   (plugin/trtt_3D_projectors.c:265-275)
 * Cubic mode: (left-c) * scl                        (plugin/trtt_3D_projectors_cubic.c:253-254) */
static void start3d(const orc_model *md, double left, double c, double h,
                    double scl, double step, double coord0, double *start,
                    double *inc)
{
  if (md->table) {
    double s = scl / step;
    *start = ((left - c) - h * coord0) * s;
    *inc = s;
  } else {
    *start = (left - c) * scl;
    *inc = scl;
  }
}

/* ------------------------------------------------------------------------ */
/* 3D parallel beam (plugin/trtt_3D_projectors.c:959-1075,                   */
/*                   plugin/trtt_3D_projectors_cubic.c:506-618)              */
/* ------------------------------------------------------------------------ */
static int parallel3d(const orc_model *md, double *out, double *in, long nx,
                      long ny, long nz, double s_scl, int s_deg, double step,
                      double coord0, long nu, long nv, double u_scl,
                      double v_scl, const double *xos, const double *xsd,
                      int job)
{
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  double a1inv = -1.0 * (1.0 / a1);
  double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  double v_x = b1 * o5 + b2 * o9, u_x = c1 * o5 + c2 * o9;
  double v_y = b1 * o6 + b2 * o10, u_y = c1 * o6 + c2 * o10;
  double v_z = b1 * o7 + b2 * o11, u_z = c1 * o7 + c2 * o11;
  double v_c = b1 * o8 + b2 * o12 + b3, u_c = c1 * o8 + c2 * o12 + c3;
  double a1sqr = a1 * a1;
  double a5sqr = v_scl * v_scl * a5 * a5;
  double a9sqr = u_scl * u_scl * a9 * a9;
  double delta_u = sqrt(1.0 + (a9sqr / (a1sqr + a5sqr)));
  double delta_v = sqrt(1.0 + (a5sqr / a1sqr));
  double rho0 = s_scl * s_scl * s_scl * delta_u * delta_v;
  double h_u = s_scl / u_scl, h_v = s_scl / v_scl;
  double scl_u = 1.0 / h_u, scl_v = 1.0 / h_v;
  double hs0 = 0.5 * (s_deg + 1);
  double hs_u = hs0 * h_u, hs_v = hs0 * h_v;
  long i, j, k;
  double *wu = (double *)malloc(sizeof(double) * (size_t)(nu > 0 ? nu : 1));
  if (wu == NULL) return ORC_FAILURE;

  for (k = 0; k < nz; ++k) {
    double vk = v_z * k + v_c, uk = u_z * k + u_c;
    for (j = 0; j < ny; ++j) {
      double vkj = vk + v_y * j, ukj = uk + u_y * j;
      for (i = 0; i < nx; ++i) {
        double vc = vkj + v_x * i, uc = ukj + u_x * i;
        double ul = clamp_left(uc - hs_u, nu), ur = clamp_right(uc + hs_u, nu - 1);
        double vl = clamp_left(vc - hs_v, nv), vr = clamp_right(vc + hs_v, nv - 1);
        double su, iu, sv, iv;
        start3d(md, ul, uc, h_u, scl_u, step, coord0, &su, &iu);
        start3d(md, vl, vc, h_v, scl_v, step, coord0, &sv, &iv);
        if (job == 0) {
          burn3d(md, 0, out, in[(k * ny + j) * nx + i], NULL, ul, ur, vl, vr, nu,
                 rho0, su, iu, sv, iv, wu);
        } else {
          burn3d(md, 1, in, 0.0, out + (k * ny + j) * nx + i, ul, ur, vl, vr,
                 nu, rho0, su, iu, sv, iv, wu);
        }
      }
    }
  }
  free(wu);
  return ORC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* 3D cone beam (plugin/trtt_3D_projectors.c:1179-1338,                      */
/*               plugin/trtt_3D_projectors_cubic.c:623-778)                  */
/* ------------------------------------------------------------------------ */
static int cone3d(const orc_model *md, double *out, double *in, long nx,
                  long ny, long nz, double s_scl, int s_deg, double step,
                  double coord0, long nu, long nv, double u_scl, double v_scl,
                  const double *xos, const double *xsd, int job)
{
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o1 = xos[0], o2 = xos[1], o3 = xos[2], o4 = xos[3];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  double a1inv = -1.0 * (1.0 / a1);
  double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  double nv_x = b1 * o5 + b2 * o9, nu_x = c1 * o5 + c2 * o9;
  double nv_y = b1 * o6 + b2 * o10, nu_y = c1 * o6 + c2 * o10;
  double nv_z = b1 * o7 + b2 * o11, nu_z = c1 * o7 + c2 * o11;
  double nv_c = b1 * o8 + b2 * o12, nu_c = c1 * o8 + c2 * o12;
  double d_x = a1 * o1 + a2 * o5 + a3 * o9;
  double d_y = a1 * o2 + a2 * o6 + a3 * o10;
  double d_z = a1 * o3 + a2 * o7 + a3 * o11;
  double d_c = a1 * o4 + a2 * o8 + a3 * o12;
  double a4sqr = a4 * a4, a4m = -1.0 * a4;
  double rho0_init = s_scl * s_scl * s_scl;
  double h_u0 = s_scl / u_scl, h_v0 = s_scl / v_scl;
  double hs0 = 0.5 * (s_deg + 1);
  long i, j, k;
  double *wu = (double *)malloc(sizeof(double) * (size_t)(nu > 0 ? nu : 1));
  if (wu == NULL) return ORC_FAILURE;

  for (k = 0; k < nz; ++k) {
    double wk1 = o3 * k + o4, nuk = nu_z * k + nu_c;
    double nvk = nv_z * k + nv_c, dk = d_z * k + d_c;
    for (j = 0; j < ny; ++j) {
      double wk2 = wk1 + o2 * j, nukj = nuk + nu_y * j;
      double nvkj = nvk + nv_y * j, dkj = dk + d_y * j;
      for (i = 0; i < nx; ++i) {
        double wk = wk2 + o1 * i;
        double num_u = nukj + nu_x * i, num_v = nvkj + nv_x * i;
        double den = dkj + d_x * i;
        double q = a4m / den;
        double uc = q * num_u + c3, vc = q * num_v + b3;
        double uca12, vca8, vca8sqr, magn, delta_u, delta_v, rho0;
        double h_u, h_v, scl_u, scl_v, ul, ur, vl, vr, su, iu, sv, iv;
        if (wk == 0) {
          fprintf(stderr, "orc_CB3D: voxel (%ld,%ld,%ld) lies in the source plane\n",
                  i, j, k);
          free(wu);
          return ORC_FAILURE;
        }
        uca12 = (uc - a12) * u_scl;
        vca8 = (vc - a8) * v_scl;
        vca8sqr = vca8 * vca8;
        magn = a4m / wk;
        delta_u = sqrt(1.0 + ((uca12 * uca12) / (a4sqr + vca8sqr)));
        delta_v = sqrt(1.0 + ((vca8sqr) / (a4sqr)));
        rho0 = rho0_init * (magn * magn) * delta_u * delta_v;
        h_u = h_u0 * magn * delta_u;
        h_v = h_v0 * magn * delta_v;
        scl_u = 1.0 / h_u;
        scl_v = 1.0 / h_v;
        ul = clamp_left(uc - hs0 * h_u, nu);
        ur = clamp_right(uc + hs0 * h_u, nu - 1);
        vl = clamp_left(vc - hs0 * h_v, nv);
        vr = clamp_right(vc + hs0 * h_v, nv - 1);
        start3d(md, ul, uc, h_u, scl_u, step, coord0, &su, &iu);
        start3d(md, vl, vc, h_v, scl_v, step, coord0, &sv, &iv);
        if (job == 0) {
          burn3d(md, 0, out, in[(k * ny + j) * nx + i], NULL, ul, ur, vl, vr, nu,
                 rho0, su, iu, sv, iv, wu);
        } else {
          burn3d(md, 1, in, 0.0, out + (k * ny + j) * nx + i, ul, ur, vl, vr,
                 nu, rho0, su, iu, sv, iv, wu);
        }
      }
    }
  }
  free(wu);
  return ORC_SUCCESS;
}

int orc_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
             int s_deg, double *footprint, double *cum_footprint,
             long size_footprint, double step_footprint, double *coord_footprint,
             long nu, long nv, double u_scl, double v_scl, double *xos,
             double *xsd, int job)
{
  orc_model md = {1, cum_footprint, size_footprint};
  (void)footprint;
  return parallel3d(&md, out, in, nx, ny, nz, s_scl, s_deg, step_footprint,
                    coord_footprint[0], nu, nv, u_scl, v_scl, xos, xsd, job);
}

int orc_PB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                   double s_scl, int s_deg, long nu, long nv, double u_scl,
                   double v_scl, double *xos, double *xsd, int job)
{
  orc_model md = {0, NULL, 0};
  return parallel3d(&md, out, in, nx, ny, nz, s_scl, s_deg, 1.0, 0.0, nu, nv,
                    u_scl, v_scl, xos, xsd, job);
}

int orc_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
             int s_deg, double *footprint, double *cum_footprint,
             long size_footprint, double step_footprint, double *coord_footprint,
             long nu, long nv, double u_scl, double v_scl, double *xos,
             double *xsd, int job)
{
  orc_model md = {1, cum_footprint, size_footprint};
  (void)footprint;
  return cone3d(&md, out, in, nx, ny, nz, s_scl, s_deg, step_footprint,
                coord_footprint[0], nu, nv, u_scl, v_scl, xos, xsd, job);
}

int orc_CB3D_cubic(double *out, double *in, long nx, long ny, long nz,
                   double s_scl, int s_deg, long nu, long nv, double u_scl,
                   double v_scl, double *xos, double *xsd, int job)
{
  orc_model md = {0, NULL, 0};
  return cone3d(&md, out, in, nx, ny, nz, s_scl, s_deg, 1.0, 0.0, nu, nv,
                u_scl, v_scl, xos, xsd, job);
}

/* ------------------------------------------------------------------------ */
/* 3D distance-driven, parallel beam (plugin/trtt_3D_projectors.c:1077-1173) */
/* ------------------------------------------------------------------------ */

/* Rectangle-overlap lengths of detector cells along one axis
 * (plugin/trtt_3D_projectors.c:443-475).  When BROKEN_FILL is set the
 * cells fully inside the rectangle all write the same slot, reproducing the
 * transpose routine of the reference (plugin/trtt_3D_projectors.c:903-917,
 * where the slot index is not advanced). */
static void dd_lengths(double b1, double b2, double scl, double *c,
                       int broken_fill)
{
  double up = ceil(b1), down = floor(b2);
  long n = (long)(down - up);
  if (n >= 0.0) {
    long s = 0, t;
    if (up > b1) c[s++] = scl * (up - b1);
    for (t = (long)up; t < down; ++t) {
      c[s] = scl;
      if (!broken_fill) ++s;
    }
    if (down < b2) c[s] = scl * (b2 - down);
  } else {
    c[0] = scl * (b2 - b1);
  }
}

int orc_DD_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                long nu, long nv, double u_scl, double v_scl, double *xos,
                double *xsd, int job)
{
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  double a1inv = -1.0 * (1.0 / a1);
  double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  double v_x = b1 * o5 + b2 * o9, u_x = c1 * o5 + c2 * o9;
  double v_y = b1 * o6 + b2 * o10, u_y = c1 * o6 + c2 * o10;
  double v_z = b1 * o7 + b2 * o11, u_z = c1 * o7 + c2 * o11;
  double v_c = b1 * o8 + b2 * o12 + b3, u_c = c1 * o8 + c2 * o12 + c3;
  double Du = fabs(u_z);
  double Dv = (fabs(v_y) > fabs(v_x)) ? fabs(v_y) : fabs(v_x);
  double h_norm = (s_scl * s_scl * s_scl) / (u_scl * v_scl * Du * Dv);
  long i, j, k;
  size_t cap = (size_t)((nu > nv ? nu : nv) + 2);
  double *cu = (double *)malloc(sizeof(double) * cap);
  double *cv = (double *)malloc(sizeof(double) * cap);
  if (cu == NULL || cv == NULL) {
    free(cu);
    free(cv);
    return ORC_FAILURE;
  }
  Du = 0.5 * Du;
  Dv = 0.5 * Dv;
  for (k = 0; k < nz; ++k) {
    double vk = v_z * k + v_c, uk = u_z * k + u_c;
    for (j = 0; j < ny; ++j) {
      double vkj = vk + v_y * j, ukj = uk + u_y * j;
      for (i = 0; i < nx; ++i) {
        double vc = vkj + v_x * i, uc = ukj + u_x * i;
        double ub1 = uc - Du, vb1 = vc - Dv, ub2 = uc + Du, vb2 = vc + Dv;
        double ulf, vlf;
        long npu, npv, base, l, m;
        double lastu = (double)(nu - 1), lastv = (double)(nv - 1);
        /* TRTT_MIN(TRTT_MAX(b,0),n-1) (plugin/trtt_3D_projectors.c:1151-1155) */
        ub1 = ub1 >= 0 ? ub1 : 0; ub1 = ub1 <= lastu ? ub1 : lastu;
        ub2 = ub2 >= 0 ? ub2 : 0; ub2 = ub2 <= lastu ? ub2 : lastu;
        vb1 = vb1 >= 0 ? vb1 : 0; vb1 = vb1 <= lastv ? vb1 : lastv;
        vb2 = vb2 >= 0 ? vb2 : 0; vb2 = vb2 <= lastv ? vb2 : lastv;
        ulf = floor(ub1);
        vlf = floor(vb1);
        base = (long)vlf * nu + (long)ulf;
        npu = (long)(ceil(ub2) - ulf);
        npv = (long)(ceil(vb2) - vlf);
        if (!(npu > 0.0 && npv > 0.0)) continue;
        memset(cu, 0, sizeof(double) * (size_t)npu);
        memset(cv, 0, sizeof(double) * (size_t)npv);
        dd_lengths(ub1, ub2, u_scl, cu, 0);
        dd_lengths(vb1, vb2, v_scl, cv, job != 0);
        if (job == 0) {
          double vox = in[(k * ny + j) * nx + i];
          for (m = 0; m < npv; ++m)
            for (l = 0; l < npu; ++l)
              out[base + m * nu + l] += h_norm * cv[m] * cu[l] * vox;
        } else {
          double *acc = out + (k * ny + j) * nx + i;
          for (m = 0; m < npv; ++m)
            for (l = 0; l < npu; ++l)
              *acc += h_norm * cv[m] * cu[l] * in[base + m * nu + l];
        }
      }
    }
  }
  free(cu);
  free(cv);
  return ORC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* 3D distance-driven, cone beam                                             */
/* ------------------------------------------------------------------------ */

/* The reference carries trtt_DD_CB3D commented out and unfinished
 * (plugin/trtt_3D_projectors.c:1340-1434): it derives the cone-beam
 * coefficients of trtt_CB3D (num_u, num_v, den, wk), declares the
 * projections of four corners of a voxel section (num_u_bb, _ub, _bu, _uu
 * and likewise num_v, den), picks the section direction x or y as
 * trtt_DD_PB3D does (|v_y| > |v_x|, with v_x = b1 o5 + b2 o9 = num_v_x),
 * clamps the footprint corners to the detector exactly like trtt_DD_PB3D
 * (:1395-1402) and burns them with the distance-driven footprint routines
 * (:1405-1425), but never computes uc, vc, Du, Dv or h_norm.  This
 * restatement completes it with the evident intent:
 *  - the section through the voxel centre perpendicular to the x axis
 *    (direction 2: corners (i, j -+ 1/2, k -+ 1/2)) or to the y axis
 *    (direction 1: (i -+ 1/2, j, k -+ 1/2)); its four corners are projected
 *    from the source with the cone-beam formula of trtt_CB3D,
 *    u = (-a4/den) num_u + c3, v = (-a4/den) num_v + b3;
 *  - the footprint is the smallest detector rectangle holding the four
 *    projected corners, ub1..ub2 x vb1..vb2;
 *  - h_norm = s^3 magn^2 delta_u delta_v / (u_scl v_scl Du Dv), Du = ub2-ub1
 *    and Dv = vb2-vb1 before clamping, magn, delta_u, delta_v those of
 *    trtt_CB3D at the voxel centre: the voxel's cone-beam detector integral
 *    (mass x magn^2 / cos(gamma), the integral trtt_CB3D's rho0 carries) is
 *    spread uniformly over its projected section, as trtt_DD_PB3D spreads
 *    the mass in parallel beam; as the source recedes the footprints and
 *    weights tend to trtt_DD_PB3D's;
 *  - the transpose accumulates the same weights as the direct projector
 *    (the adjoint); the transpose routine of trtt_DD_PB3D writes every
 *    fully covered v cell into one slot (:915), which is not carried over
 *    to this unfinished projector.
 * A voxel centre in the source plane (wk == 0) fails as in trtt_CB3D; a
 * section corner in the source plane or a degenerate footprint (Du Dv == 0)
 * gives no contribution. */
int orc_DD_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl,
                long nu, long nv, double u_scl, double v_scl, double *xos,
                double *xsd, int job)
{
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o1 = xos[0], o2 = xos[1], o3 = xos[2], o4 = xos[3];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  double a1inv = -1.0 * (1.0 / a1);
  double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  double nv_x = b1 * o5 + b2 * o9, nu_x = c1 * o5 + c2 * o9;
  double nv_y = b1 * o6 + b2 * o10, nu_y = c1 * o6 + c2 * o10;
  double nv_z = b1 * o7 + b2 * o11, nu_z = c1 * o7 + c2 * o11;
  double nv_c = b1 * o8 + b2 * o12, nu_c = c1 * o8 + c2 * o12;
  double d_x = a1 * o1 + a2 * o5 + a3 * o9;
  double d_y = a1 * o2 + a2 * o6 + a3 * o10;
  double d_z = a1 * o3 + a2 * o7 + a3 * o11;
  double d_c = a1 * o4 + a2 * o8 + a3 * o12;
  double a4sqr = a4 * a4, a4m = -1.0 * a4;
  double s3 = s_scl * s_scl * s_scl;
  int axis = (fabs(nv_y) > fabs(nv_x)) ? 2 : 1;
  long i, j, k;
  size_t cap = (size_t)((nu > nv ? nu : nv) + 2);
  double *cu = (double *)malloc(sizeof(double) * cap);
  double *cv = (double *)malloc(sizeof(double) * cap);
  if (cu == NULL || cv == NULL) {
    free(cu);
    free(cv);
    return ORC_FAILURE;
  }
  for (k = 0; k < nz; ++k) {
    for (j = 0; j < ny; ++j) {
      for (i = 0; i < nx; ++i) {
        double x = (double)i, y = (double)j, z = (double)k;
        double wk = o1 * x + o2 * y + o3 * z + o4;
        double ucor[4], vcor[4];
        double num_u, num_v, den, q, uc, vc, magn, vca8sqr, dv, du;
        double ub1, ub2, vb1, vb2, Du, Dv, h_norm, ulf, vlf;
        double lastu = (double)(nu - 1), lastv = (double)(nv - 1);
        long npu, npv, base, l, m;
        int c, bad = 0;
        if (wk == 0.0) {
          free(cu);
          free(cv);
          fprintf(stderr, "orc_DD_CB3D: voxel in the source plane\n");
          return ORC_FAILURE;
        }
        /* corners bb, ub, bu, uu: (section axis -, z -), (+, -), (-, +), (+, +) */
        for (c = 0; c < 4; ++c) {
          double hs = (c & 1) ? 0.5 : -0.5, hz = (c & 2) ? 0.5 : -0.5;
          double cx = x + (axis == 1 ? hs : 0.0), cy = y + (axis == 2 ? hs : 0.0);
          double cz = z + hz;
          double nu_ = nu_x * cx + nu_y * cy + nu_z * cz + nu_c;
          double nv_ = nv_x * cx + nv_y * cy + nv_z * cz + nv_c;
          double de = d_x * cx + d_y * cy + d_z * cz + d_c;
          double qc = a4m / de;
          ucor[c] = qc * nu_ + c3;
          vcor[c] = qc * nv_ + b3;
          if (!(isfinite(ucor[c]) && isfinite(vcor[c]))) bad = 1;
        }
        if (bad) continue;
        ub1 = ub2 = ucor[0];
        vb1 = vb2 = vcor[0];
        for (c = 1; c < 4; ++c) {
          ub1 = ucor[c] < ub1 ? ucor[c] : ub1;
          ub2 = ucor[c] > ub2 ? ucor[c] : ub2;
          vb1 = vcor[c] < vb1 ? vcor[c] : vb1;
          vb2 = vcor[c] > vb2 ? vcor[c] : vb2;
        }
        Du = ub2 - ub1;
        Dv = vb2 - vb1;
        /* magnification and obliquity at the centre (trtt_CB3D :1253-1280) */
        num_u = nu_x * x + nu_y * y + nu_z * z + nu_c;
        num_v = nv_x * x + nv_y * y + nv_z * z + nv_c;
        den = d_x * x + d_y * y + d_z * z + d_c;
        q = a4m / den;
        uc = q * num_u + c3;
        vc = q * num_v + b3;
        magn = a4m / wk;
        vca8sqr = ((vc - a8) * v_scl) * ((vc - a8) * v_scl);
        dv = sqrt(1.0 + vca8sqr / a4sqr);
        du = sqrt(1.0 + (((uc - a12) * u_scl) * ((uc - a12) * u_scl)) / (a4sqr + vca8sqr));
        h_norm = (s3 * (magn * magn) * du * dv) / (u_scl * v_scl * Du * Dv);
        if (!isfinite(h_norm)) continue;
        /* TRTT_MIN(TRTT_MAX(b,0),n-1) (plugin/trtt_3D_projectors.c:1395-1402) */
        ub1 = ub1 >= 0 ? ub1 : 0; ub1 = ub1 <= lastu ? ub1 : lastu;
        ub2 = ub2 >= 0 ? ub2 : 0; ub2 = ub2 <= lastu ? ub2 : lastu;
        vb1 = vb1 >= 0 ? vb1 : 0; vb1 = vb1 <= lastv ? vb1 : lastv;
        vb2 = vb2 >= 0 ? vb2 : 0; vb2 = vb2 <= lastv ? vb2 : lastv;
        ulf = floor(ub1);
        vlf = floor(vb1);
        base = (long)vlf * nu + (long)ulf;
        npu = (long)(ceil(ub2) - ulf);
        npv = (long)(ceil(vb2) - vlf);
        if (!(npu > 0.0 && npv > 0.0)) continue;
        memset(cu, 0, sizeof(double) * (size_t)npu);
        memset(cv, 0, sizeof(double) * (size_t)npv);
        dd_lengths(ub1, ub2, u_scl, cu, 0);
        dd_lengths(vb1, vb2, v_scl, cv, 0);
        if (job == 0) {
          double vox = in[(k * ny + j) * nx + i];
          for (m = 0; m < npv; ++m)
            for (l = 0; l < npu; ++l)
              out[base + m * nu + l] += h_norm * cv[m] * cu[l] * vox;
        } else {
          double *acc = out + (k * ny + j) * nx + i;
          for (m = 0; m < npv; ++m)
            for (l = 0; l < npu; ++l)
              *acc += h_norm * cv[m] * cu[l] * in[base + m * nu + l];
        }
      }
    }
  }
  free(cu);
  free(cv);
  return ORC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* 2D projectors                                                             */
/* ------------------------------------------------------------------------ */

/* One pixel of a 2D projector.  direct: out[v] += (rho0*vox)*w (table) or
 * (w*vox)*rho0 (cubic); transpose: acc += (rho0*pix[v])*w
 * (plugin/trtt_2D_projectors.c:71-171, plugin/trtt_2D_projectors_cubic.c:99-194). */
static void burn2d(const orc_model *md, int job, double *pix, double vox,
                   double *acc, double vl, double vr, double rho0,
                   double start, double inc)
{
  long i, n, id = (long)vl;
  double p0;
  if (!(vl < vr)) return;
  n = (long)(vr - vl);
  p0 = model_primitive(md, start);
  for (i = 0; i < n; ++i) {
    double x = start + (i + 1) * inc;
    double p1 = model_primitive(md, x);
    if (job == 0) {
      if (md->table) pix[id + i] += rho0 * vox * (p1 - p0);
      else pix[id + i] += (p1 - p0) * vox * rho0;
    } else {
      *acc += rho0 * pix[id + i] * (p1 - p0);
    }
    p0 = p1;
  }
}

/* Normalised start of a 2D footprint.
 * Table: (vl - (vc + coord0*h)) * scl   (plugin/trtt_2D_projectors.c:94-97)
 * Cubic: (vl - vc) * scl                (plugin/trtt_2D_projectors_cubic.c:119) */
static double start2d(const orc_model *md, double vl, double vc, double h,
                      double scl, double coord0)
{
  if (md->table) return (vl - (vc + coord0 * h)) * scl;
  return (vl - vc) * scl;
}

/* Parallel-beam 2D constants (plugin/trtt_2D_projectors.c:190-218). */
typedef struct {
  double b1o5, b1o6, b1o8b3, rho0, h, scl, hs;
} par2d_t;

static void par2d_setup(par2d_t *g, const orc_model *md, double s_scl,
                        int s_deg, double step, double v_scl,
                        const double *xos, const double *xsd)
{
  double a1 = xsd[0];
  double a1inv = -1.0 * (1.0 / a1);
  double a2 = xsd[1], a4 = xsd[3], a5 = xsd[4];
  double a5a1 = a5 * a1inv;
  double a5a1scl = a5a1 * v_scl;
  double a6 = xsd[5], a8 = xsd[7];
  double b1 = a6 + a5a1 * a2;
  double b3 = a8 + a5a1 * a4;
  double delta_v = sqrt(1 + a5a1scl * a5a1scl);
  g->b1o5 = b1 * xos[4];
  g->b1o6 = b1 * xos[5];
  g->b1o8b3 = b1 * xos[7] + b3;
  g->rho0 = s_scl * s_scl * delta_v;
  g->h = (delta_v * s_scl) / v_scl;
  g->scl = md->table ? 1 / (g->h * step) : 1 / g->h;
  g->hs = 0.5 * (s_deg + 1) * g->h;
}

/* Fan-beam 2D constants (plugin/trtt_2D_projectors.c:277-315). */
typedef struct {
  double a4m, a4sqr, a8, b3, b1o5, b1o6, b1o8, d_x, d_y, d_c;
  double rho0_init, h_init, hs0;
} fan2d_t;

static void fan2d_setup(fan2d_t *g, double s_scl, int s_deg, double v_scl,
                        const double *xos, const double *xsd)
{
  double a1 = xsd[0];
  double a1inv = -1.0 * (1.0 / a1);
  double a2 = xsd[1], a4 = xsd[3], a5 = xsd[4], a6 = xsd[5], a8 = xsd[7];
  double b1 = a6 + a1inv * a5 * a2;
  g->a4m = -1.0 * a4;
  g->a4sqr = a4 * a4;
  g->a8 = a8;
  g->b3 = a8 + a1inv * a5 * a4;
  g->b1o5 = b1 * xos[4];
  g->b1o6 = b1 * xos[5];
  g->b1o8 = b1 * xos[7];
  g->d_x = a1 * xos[0] + a2 * xos[4];
  g->d_y = a1 * xos[1] + a2 * xos[5];
  g->d_c = a1 * xos[3] + a2 * xos[7];
  g->rho0_init = s_scl * s_scl;
  g->h_init = s_scl / v_scl;
  g->hs0 = 0.5 * (s_deg + 1);
}

/* Fan-beam per-pixel geometry (plugin/trtt_2D_projectors.c:330-352).
 * Returns 0 on success, -1 if the pixel lies on the source line. */
static int fan2d_pixel(const fan2d_t *g, const orc_model *md, double step,
                       double v_scl, const double *xos, long i, long j,
                       double *vc, double *rho0, double *h, double *scl,
                       double *hs)
{
  double wk = (xos[1] * j + xos[3]) + xos[0] * i;
  double num = (g->b1o6 * j + g->b1o8) + g->b1o5 * i;
  double den = (g->d_y * j + g->d_c) + g->d_x * i;
  double magn, vca8, delta_v;
  *vc = (g->a4m / den) * num + g->b3;
  if (wk == 0) return ORC_FAILURE;
  magn = g->a4m / wk;
  vca8 = (*vc - g->a8) * v_scl;
  delta_v = sqrt(1.0 + ((vca8 * vca8) / (g->a4sqr)));
  *rho0 = g->rho0_init * magn * delta_v;
  *h = g->h_init * magn * delta_v;
  *scl = md->table ? 1 / (*h * step) : 1.0 / *h;
  *hs = g->hs0 * *h;
  return ORC_SUCCESS;
}

static int parallel2d(const orc_model *md, double *out, double *in, long nx,
                      long ny, double s_scl, int s_deg, double step,
                      double coord0, long nv, double v_scl, const double *xos,
                      const double *xsd, int job)
{
  par2d_t g;
  long i, j, right_max = md->table ? nv - 1 : nv - 2;
  par2d_setup(&g, md, s_scl, s_deg, step, v_scl, xos, xsd);
  for (j = 0; j < ny; ++j) {
    double vj = g.b1o6 * j + g.b1o8b3;
    for (i = 0; i < nx; ++i) {
      double vc = vj + g.b1o5 * i;
      double vl = clamp_left(vc - g.hs, nv), vr = clamp_right(vc + g.hs, right_max);
      double st = start2d(md, vl, vc, g.h, g.scl, coord0);
      if (job == 0) burn2d(md, 0, out, in[j * nx + i], NULL, vl, vr, g.rho0, st, g.scl);
      else burn2d(md, 1, in, 0.0, out + j * nx + i, vl, vr, g.rho0, st, g.scl);
    }
  }
  return ORC_SUCCESS;
}

static int fan2d(const orc_model *md, double *out, double *in, long nx, long ny,
                 double s_scl, int s_deg, double step, double coord0, long nv,
                 double v_scl, const double *xos, const double *xsd, int job)
{
  fan2d_t g;
  long i, j, right_max = md->table ? nv - 1 : nv - 2;
  fan2d_setup(&g, s_scl, s_deg, v_scl, xos, xsd);
  for (j = 0; j < ny; ++j) {
    for (i = 0; i < nx; ++i) {
      double vc, rho0, h, scl, hs, vl, vr, st;
      if (fan2d_pixel(&g, md, step, v_scl, xos, i, j, &vc, &rho0, &h, &scl, &hs)) {
        fprintf(stderr, "orc_FB2D: pixel (%ld,%ld) lies on the source line\n", i, j);
        return ORC_FAILURE;
      }
      vl = clamp_left(vc - hs, nv);
      vr = clamp_right(vc + hs, right_max);
      st = start2d(md, vl, vc, h, scl, coord0);
      if (job == 0) burn2d(md, 0, out, in[j * nx + i], NULL, vl, vr, rho0, st, scl);
      else burn2d(md, 1, in, 0.0, out + j * nx + i, vl, vr, rho0, st, scl);
    }
  }
  return ORC_SUCCESS;
}

int orc_PB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
             double *footprint, double *cum_footprint, long size_footprint,
             double step_footprint, double *coord_footprint, long nv,
             double v_scl, double *xos, double *xsd, int job)
{
  orc_model md = {1, cum_footprint, size_footprint};
  (void)footprint;
  return parallel2d(&md, out, in, nx, ny, s_scl, s_deg, step_footprint,
                    coord_footprint[0], nv, v_scl, xos, xsd, job);
}

int orc_FB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
             double *footprint, double *cum_footprint, long size_footprint,
             double step_footprint, double *coord_footprint, long nv,
             double v_scl, double *xos, double *xsd, int job)
{
  orc_model md = {1, cum_footprint, size_footprint};
  (void)footprint;
  return fan2d(&md, out, in, nx, ny, s_scl, s_deg, step_footprint,
               coord_footprint[0], nv, v_scl, xos, xsd, job);
}

int orc_PB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                   int s_deg, long nv, double v_scl, double *xos, double *xsd,
                   int job)
{
  orc_model md = {0, NULL, 0};
  return parallel2d(&md, out, in, nx, ny, s_scl, s_deg, 1.0, 0.0, nv, v_scl,
                    xos, xsd, job);
}

int orc_FB2D_cubic(double *out, double *in, long nx, long ny, double s_scl,
                   int s_deg, long nv, double v_scl, double *xos, double *xsd,
                   int job)
{
  orc_model md = {0, NULL, 0};
  return fan2d(&md, out, in, nx, ny, s_scl, s_deg, 1.0, 0.0, nv, v_scl, xos,
               xsd, job);
}

int orc_PB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                     int s_deg, double *footprint, double *cum_footprint,
                     long size_footprint, double step_footprint,
                     double *coord_footprint, long nv, double v_scl,
                     double *xos, double *xsd)
{
  orc_model md = {1, cum_footprint, size_footprint};
  par2d_t g;
  double vc, vl, vr;
  (void)footprint; (void)nx; (void)ny;
  par2d_setup(&g, &md, s_scl, s_deg, step_footprint, v_scl, xos, xsd);
  vc = g.b1o6 * j + g.b1o8b3 + g.b1o5 * i;
  vl = clamp_left(vc - g.hs, nv);
  vr = clamp_right(vc + g.hs, nv - 1);
  burn2d(&md, 0, out, 1.0, NULL, vl, vr, g.rho0,
         start2d(&md, vl, vc, g.h, g.scl, coord_footprint[0]), g.scl);
  return ORC_SUCCESS;
}

int orc_FB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl,
                     int s_deg, double *footprint, double *cum_footprint,
                     long size_footprint, double step_footprint,
                     double *coord_footprint, long nv, double v_scl,
                     double *xos, double *xsd)
{
  orc_model md = {1, cum_footprint, size_footprint};
  fan2d_t g;
  double vc, rho0, h, scl, hs, vl, vr;
  (void)footprint; (void)nx; (void)ny;
  fan2d_setup(&g, s_scl, s_deg, v_scl, xos, xsd);
  if (fan2d_pixel(&g, &md, step_footprint, v_scl, xos, i, j, &vc, &rho0, &h, &scl, &hs)) {
    fprintf(stderr, "orc_FB2D_sparser: pixel (%ld,%ld) lies on the source line\n", i, j);
    return ORC_FAILURE;
  }
  vl = clamp_left(vc - hs, nv);
  vr = clamp_right(vc + hs, nv - 1);
  burn2d(&md, 0, out, 1.0, NULL, vl, vr, rho0,
         start2d(&md, vl, vc, h, scl, coord_footprint[0]), scl);
  return ORC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* Sparse matrix-vector product, 1-based COO (plugin/trtt_common.c:62-69)   */
/* ------------------------------------------------------------------------ */
int orc_mvmult(double *out, double *in, long number, double *a, long *i, long *j)
{
  long k;
  for (k = 0; k < number; ++k) out[i[k] - 1] += a[k] * in[j[k] - 1];
  return ORC_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* Long-Fessler separable footprint, fan beam                                */
/* (tomography-LongFessler-model/LongFessler2D.c:29-681)                      */
/* ------------------------------------------------------------------------ */

static double lf_tri(double a, double b, double c)
{
  if (a >= b) return 0.0;
  return (b + a) * (b - a) / (c + c);
}
static double lf_rect(double a, double b)
{
  if (a >= b) return 0.0;
  return (b - a);
}
static double lf_max(double a, double b) { return a >= b ? a : b; }
static double lf_min(double a, double b) { return a <= b ? a : b; }

/* Per-view constants (LongFessler2D.c:61-76). */
typedef struct {
  double cb, sb, x0, y0, off, scale, size, vs, ps, sd;
  long n1, n2, nd;
} lf_view;

static void lf_setup(lf_view *g, const orc_lf2d_parameters *p, double beta,
                     double detector_offset)
{
  double off_y, off_x;
  g->cb = cos(beta);
  g->sb = sin(beta);
  off_y = g->cb * (p->objectOffset1) + g->sb * (p->objectOffset2);
  off_x = -g->sb * (p->objectOffset1) + g->cb * (p->objectOffset2);
  g->n1 = p->objectDimension1;
  g->n2 = p->objectDimension2;
  g->nd = p->detectorDimension;
  g->vs = p->voxelSize;
  g->ps = p->pixelSize;
  g->sd = p->sourceDistance;
  g->x0 = off_x - 0.5 * (g->n1 - 1) * g->vs;
  g->y0 = off_y - 0.5 * (g->n2 - 1) * g->vs;
  g->off = detector_offset / p->pixelStep + 0.5 * (g->nd - 1);
  g->scale = (p->sourceDistance + p->detectorDistance) / p->pixelStep;
  g->size = p->pixelSize / p->pixelStep;
}

/* Sorted trapezoid corners t[0..3], obliquity factor sqrt(1+q^2) and the
 * impacted cell range of voxel (i1,i2) (LongFessler2D.c:90-125). */
static void lf_voxel(const lf_view *g, long i1, long i2, double t[4],
                     double *obliq, long *kf, long *kl)
{
  double y = g->y0 + i2 * g->vs;
  double y1 = y - 0.5 * g->vs, y2 = y + 0.5 * g->vs;
  double x = g->x0 + i1 * g->vs;
  double x1 = x - 0.5 * g->vs, x2 = x + 0.5 * g->vs;
  double qx, qy, q, tmp;
#define LF_S(X, Y) (g->scale * ((Y) * g->sb + (X) * g->cb) / (g->sd - ((Y) * g->cb - (X) * g->sb)) + g->off)
  t[0] = LF_S(x1, y1);
  t[1] = LF_S(x2, y1);
  t[2] = LF_S(x1, y2);
  t[3] = LF_S(x2, y2);
#undef LF_S
#define LF_SWAP(a, b) if (t[a] > t[b]) { tmp = t[a]; t[a] = t[b]; t[b] = tmp; }
  LF_SWAP(0, 1);
  LF_SWAP(2, 3);
  LF_SWAP(0, 2);
  LF_SWAP(1, 3);
  LF_SWAP(1, 2);
#undef LF_SWAP
  qx = x + g->sd * g->sb;
  qy = y - g->sd * g->cb;
  q = (fabs(qy) > fabs(qx) ? qx / qy : qy / qx);
  *obliq = sqrt(1.0 + q * q);
  *kf = (long)floor(t[0] - 0.5 * g->size);
  if (*kf < 0) *kf = 0;
  *kl = (long)ceil(t[3] + 0.5 * g->size);
  if (*kl >= g->nd) *kl = g->nd - 1;
}

/* Trapezoid integral over cell k, in cell units (LongFessler2D.c:129-136). */
static double lf_gamma(const double t[4], long k, double size)
{
  double s1 = k - 0.5 * size;
  double s2 = s1 + size;
  return (lf_tri(lf_max(s1, t[0]) - t[0], lf_min(s2, t[1]) - t[0], t[1] - t[0]) +
          lf_rect(lf_max(s1, t[1]), lf_min(s2, t[2])) +
          lf_tri(t[3] - lf_min(s2, t[3]), t[3] - lf_max(s1, t[2]), t[3] - t[2]));
}

/* Trapezoid height at cell centre k (LongFessler2D.c:226-234, :451-460). */
static double lf_line(const double t[4], long k)
{
  if (k >= t[0] && k < t[1]) return (k - t[0]) / (t[1] - t[0]);
  if (k >= t[1] && k < t[2]) return 1;
  if (k >= t[2] && k < t[3]) return (k - t[3]) / (t[2] - t[3]);
  return 0;
}

void orc_lf2d_direct(const orc_lf2d_parameters *p, double beta, double offset,
                     const double voxel[], double pixel[], int clr)
{
  lf_view g;
  long i1, i2, k, kf, kl;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(pixel, 0, sizeof(double) * (size_t)g.nd);
  for (i2 = 0; i2 < g.n2; ++i2) {
    for (i1 = 0; i1 < g.n1; ++i1) {
      double t[4], ob, alpha;
      lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
      alpha = (ob * (g.vs * g.ps) * voxel[i1 + i2 * g.n1]);
      for (k = kf; k <= kl; ++k) pixel[k] += lf_gamma(t, k, g.size) * alpha;
    }
  }
}

void orc_lf2d_line_integ_direct(const orc_lf2d_parameters *p, double beta,
                                double offset, const double voxel[],
                                double pixel[], int clr)
{
  lf_view g;
  long i1, i2, k, kf, kl;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(pixel, 0, sizeof(double) * (size_t)g.nd);
  for (i2 = 0; i2 < g.n2; ++i2) {
    for (i1 = 0; i1 < g.n1; ++i1) {
      double t[4], ob, alpha;
      lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
      alpha = (ob * g.vs * voxel[i1 + i2 * g.n1]);
      for (k = kf; k <= kl; ++k) {
        /* (alpha*(k-t0))/(t1-t0) etc., LongFessler2D.c:226-234 */
        if (k >= t[0] && k < t[1]) pixel[k] += alpha * (k - t[0]) / (t[1] - t[0]);
        else if (k >= t[1] && k < t[2]) pixel[k] += alpha;
        else if (k >= t[2] && k < t[3]) pixel[k] += alpha * (k - t[3]) / (t[2] - t[3]);
        else pixel[k] += 0;
      }
    }
  }
}

void orc_lf2d_adjoint(const orc_lf2d_parameters *p, double beta, double offset,
                      const double pixel[], double voxel[], int clr)
{
  lf_view g;
  long i1, i2, k, kf, kl;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(voxel, 0, sizeof(double) * (size_t)(g.n1 * g.n2));
  for (i2 = 0; i2 < g.n2; ++i2) {
    for (i1 = 0; i1 < g.n1; ++i1) {
      double t[4], ob, alpha, sum = 0.0;
      lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
      alpha = ob * (g.vs * g.ps);
      for (k = kf; k <= kl; ++k) sum += alpha * lf_gamma(t, k, g.size) * pixel[k];
      voxel[i1 + i2 * g.n1] += sum;
    }
  }
}

void orc_lf2d_line_integ_adjoint(const orc_lf2d_parameters *p, double beta,
                                 double offset, const double pixel[],
                                 double voxel[], int clr)
{
  lf_view g;
  long i1, i2, k, kf, kl;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(voxel, 0, sizeof(double) * (size_t)(g.n1 * g.n2));
  for (i2 = 0; i2 < g.n2; ++i2) {
    for (i1 = 0; i1 < g.n1; ++i1) {
      double t[4], ob, alpha, sum = 0.0;
      lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
      alpha = ob * g.vs;
      for (k = kf; k <= kl; ++k) sum += alpha * lf_line(t, k) * pixel[k];
      voxel[i1 + i2 * g.n1] += sum;
    }
  }
}

void orc_lf2d_sparser(const orc_lf2d_parameters *p, double beta, double offset,
                      long i1, long i2, double pixel[], int clr)
{
  lf_view g;
  long k, kf, kl;
  double t[4], ob, alpha;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(pixel, 0, sizeof(double) * (size_t)g.nd);
  lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
  alpha = (ob * (g.vs * g.ps));
  for (k = kf; k <= kl; ++k) pixel[k] += lf_gamma(t, k, g.size) * alpha;
}

void orc_lf2d_line_integ_sparser(const orc_lf2d_parameters *p, double beta,
                                 double offset, long i1, long i2,
                                 double pixel[], int clr)
{
  lf_view g;
  long k, kf, kl;
  double t[4], ob, alpha;
  lf_setup(&g, p, beta, offset);
  if (clr) memset(pixel, 0, sizeof(double) * (size_t)g.nd);
  lf_voxel(&g, i1, i2, t, &ob, &kf, &kl);
  alpha = (ob * g.vs);
  for (k = kf; k <= kl; ++k) {
    if (k >= t[0] && k < t[1]) pixel[k] += alpha * (k - t[0]) / (t[1] - t[0]);
    else if (k >= t[1] && k < t[2]) pixel[k] += alpha;
    else if (k >= t[2] && k < t[3]) pixel[k] += alpha * (k - t[3]) / (t[2] - t[3]);
    else pixel[k] += 0;
  }
}

/* ------------------------------------------------------------------------ */
/* Footprint table (Ytrtt_tomobj.i:140-196)                                  */
/* ------------------------------------------------------------------------ */

/* Centred B-spline of degree n by the two-term recursion
 *   b_n(x) = ((n+1)/2 + x)/n * b_{n-1}(x+1/2) + ((n+1)/2 - x)/n * b_{n-1}(x-1/2),
 * b_0 the unit box on [-1/2, 1/2).  The reference samples the same function
 * through an external spline package that is not part of the repository, so
 * this sampling is a restatement of the published definition. */
static double bspline(int n, double x)
{
  if (n == 0) return (x >= -0.5 && x < 0.5) ? 1.0 : 0.0;
  return ((0.5 * (n + 1) + x) * bspline(n - 1, x + 0.5) +
          (0.5 * (n + 1) - x) * bspline(n - 1, x - 0.5)) / n;
}

double orc_footprint_table(int deg, long m, double *footprint, double *cum,
                           double *coord)
{
  long n = 2 * deg + 3, i;
  double step = (double)(n - 1) / (double)(m - 1);
  for (i = 0; i < m; ++i) {
    coord[i] = (double)i * step - 0.5 * (double)(n - 1);
    footprint[i] = bspline(deg, coord[i]);
  }
  /* trapezoid partial sums (Ytrtt_tomobj.i:183-196; the Yorick loop's first
   * term reads the last table entries, which are zero) */
  cum[0] = 0.0;
  for (i = 1; i < m; ++i) cum[i] = cum[i - 1] + 0.5 * step * (footprint[i - 1] + footprint[i]);
  return step;
}
