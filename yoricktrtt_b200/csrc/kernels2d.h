// kernels2d.h -- 2D projector, Long-Fessler, distance-driven 3D and sparse
// kernels: parameter blocks and launchers (internal to libtrtt_b200).
#pragma once

#include <cuda_runtime.h>

#include "kernels.h"

namespace trtt {

// 2D B-spline projector parameters common to all views.
struct Params2D {
  int nx, ny, nv;
  int fan;    // 1: fan beam (trtt_FB2D), 0: parallel (trtt_PB2D)
  int table;  // 1: tabulated footprint, 0: closed-form cubic
  int pad_;
  double v_scl;
  double rho0_init;  // s^2
  double h_init;     // s / v_scl
  double hs0;        // (s_deg+1)/2
  const double *cum;
  double last, step, coord0;
};

// Per-view constants (plugin/trtt_2D_projectors.c:190-218 and :277-315).
struct View2D {
  // fan beam
  double o1, o2, o4;
  double a4m, a4sqr, a8, b3;
  double b1o5, b1o6, b1o8;
  double d_x, d_y, d_c;
  // parallel beam
  double b1o8b3, p_rho0, p_h, p_scl, p_hs;
};

// Long-Fessler per-view constants (LongFessler2D.c:61-76).
struct LFView {
  double cb, sb, x0, y0, off, scale, size, vs, ps, sd;
  int n1, n2, nd, pad_;
};

cudaError_t launch_fwd2d(const Params2D &P, const View2D *views, int nviews, const float *img,
                         float *sino, int *err, cudaStream_t st);
cudaError_t launch_back2d(const Params2D &P, const View2D *views, int nviews, const float *sino,
                          float *img, int *err, cudaStream_t st);
cudaError_t launch_sparser2d(const Params2D &P, const View2D *view, int i, int j, double *out,
                             int *err, cudaStream_t st);
cudaError_t launch_assemble2d(const Params2D &P, const View2D *views, int nviews, int max_cells,
                              double *a, long *rows, long *cols, int *err, cudaStream_t st);

cudaError_t launch_lf_fwd(const LFView *views, int nviews, int nd, int line, const float *img,
                          float *sino, cudaStream_t st);
cudaError_t launch_lf_back(const LFView *views, int nviews, int npix, int line, const float *sino,
                           float *img, cudaStream_t st);
cudaError_t launch_lf_sparser(const LFView *view, int line, int i1, int i2, double *out,
                              cudaStream_t st);

// Distance-driven 3D parallel beam (dd3d.cu).
struct ParamsDD {
  int nx, ny, nz, nu, nv, pad_;
  double u_scl, v_scl;
  double u_x, u_y, u_z, u_c, v_x, v_y, v_z, v_c;
  double Du, Dv, h_norm;
};
cudaError_t launch_dd_fwd(const ParamsDD &P, const double *vol, double *det, cudaStream_t st);

// Cone-beam distance-driven view (dd3d.cu): the coefficients of trtt_CB3D
// (num_u, num_v, den, wk) and the voxel-section direction (1: x, 2: y).
struct ParamsDDC {
  int nx, ny, nz, nu, nv, axis;
  double u_scl, v_scl, s3;
  double o1, o2, o3, o4;
  double nu_x, nu_y, nu_z, nu_c, nv_x, nv_y, nv_z, nv_c;
  double d_x, d_y, d_z, d_c;
  double a4m, a4sqr, a8, a12, b3, c3;
};
// views_dev: nviews device records; det: nviews images of det_stride
// doubles; err |= 1 when a voxel centre lies in the source plane.
cudaError_t launch_ddc_fwd(const ParamsDDC *views_dev, int nviews, long nvox, const double *vol,
                           double *det, long det_stride, int *err, cudaStream_t st);
cudaError_t launch_ddc_back(const ParamsDDC *views_dev, int nviews, long nvox, const double *det,
                            long det_stride, double *vol, int *err, cudaStream_t st);
cudaError_t launch_dd_back(const ParamsDD &P, const double *det, double *vol, cudaStream_t st);

// Sparse COO product out[i-1] += a * in[j-1] (spmv.cu).
cudaError_t launch_mvmult(const double *a, const long *i, const long *j, long nnz,
                          const double *in, double *out, cudaStream_t st);

}  // namespace trtt
