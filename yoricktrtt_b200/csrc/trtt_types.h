// trtt_types.h -- plain-old-data structures shared by the host runtime and
// the device kernels.  Per-view geometry coefficients are derived on the
// host in FP64 with the operand order of the reference projectors, so the
// device sees exactly the constants the reference would compute.
#pragma once

#include <cstdint>

namespace trtt {

enum Geometry3D : int { GEOM_PARALLEL = 0, GEOM_CONE = 1 };
enum FootprintModel : int { MODEL_CUBIC = 0, MODEL_TABLE = 1 };

// One view of a 3D projector (plugin/trtt_3D_projectors.c:959-1010 for
// parallel beam, :1179-1230 for cone beam).
struct View3D {
  // cone beam: wk = o1 i + o2 j + o3 k + o4 ; num_u, num_v, den likewise
  double o1, o2, o3, o4;
  double nu_x, nu_y, nu_z, nu_c;
  double nv_x, nv_y, nv_z, nv_c;
  double d_x, d_y, d_z, d_c;
  double a4m, a4sqr, a8, a12, b3, c3;
  // parallel beam: uc = u_x i + u_y j + u_z k + u_c (b3/c3 folded in)
  double u_x, u_y, u_z, u_c;
  double v_x, v_y, v_z, v_c;
  double p_rho0, p_h_u, p_h_v, p_scl_u, p_scl_v, p_hs_u, p_hs_v;
  double p_sclt_u, p_sclt_v;  // scl/step (table mode)
  // temporal interpolation (4D): the projected volume is
  // w0 * gate[g0] + w1 * gate[g1]; the transpose scatters with the same
  // weights.  Plain 3D views use g0 = g1 = 0, w0 = 1, w1 = 0.
  int g0, g1;
  float w0, w1;
  int factorized;  // 1 if the transaxial footprint does not depend on k
  int pad_;
};

// Object / detector / footprint parameters common to all views of a call.
struct Params3D {
  int geom;    // Geometry3D
  int model;   // FootprintModel
  int nx, ny, nz, nu, nv;
  int nt;      // number of gates (1 for plain 3D)
  double s_scl, u_scl, v_scl;
  double rho0_init;  // s^3
  double h_u0, h_v0; // s/u_scl, s/v_scl
  double hs0;        // (s_deg+1)/2
  // table footprint (model == MODEL_TABLE)
  const double *cum;
  double last;       // size_footprint - 1
  double step;       // step_footprint
  double coord0;     // coord_footprint[0]
  int size;          // size_footprint
  int pad_;
};

}  // namespace trtt
