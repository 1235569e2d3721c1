// abi2d.cu -- C ABI of the 2D B-spline projectors, their sparse column
// generators, the Long-Fessler model, the distance-driven 3D projector and
// the COO product: drop-in symbols (host double*, reference semantics) and
// the native 2D plan (device float*, many views per launch).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "kernels2d.h"
#include "runtime.h"
#include "trtt_b200.h"

using namespace trtt;

namespace {

// Per-view constants of the 2D projectors, reference operand order
// (parallel plugin/trtt_2D_projectors.c:190-218, fan :277-315).
void make_view2d(const Params2D &P, double s_scl, int s_deg, const double *xos,
                 const double *xsd, View2D &V)
{
  std::memset(&V, 0, sizeof(V));
  const double a1 = xsd[0];
  const double a1inv = -1.0 * (1.0 / a1);
  const double a2 = xsd[1], a4 = xsd[3], a5 = xsd[4], a6 = xsd[5], a8 = xsd[7];
  // fan beam
  const double b1 = a6 + a1inv * a5 * a2;
  V.o1 = xos[0];
  V.o2 = xos[1];
  V.o4 = xos[3];
  V.a4m = -1.0 * a4;
  V.a4sqr = a4 * a4;
  V.a8 = a8;
  V.b3 = a8 + a1inv * a5 * a4;
  V.b1o5 = b1 * xos[4];
  V.b1o6 = b1 * xos[5];
  V.b1o8 = b1 * xos[7];
  V.d_x = a1 * xos[0] + a2 * xos[4];
  V.d_y = a1 * xos[1] + a2 * xos[5];
  V.d_c = a1 * xos[3] + a2 * xos[7];
  // parallel beam
  const double a5a1 = a5 * a1inv;
  const double a5a1scl = a5a1 * P.v_scl;
  const double b1p = a6 + a5a1 * a2;
  const double b3p = a8 + a5a1 * a4;
  const double delta_v = std::sqrt(1 + a5a1scl * a5a1scl);
  if (!P.fan) {
    V.b1o5 = b1p * xos[4];
    V.b1o6 = b1p * xos[5];
  }
  V.b1o8b3 = b1p * xos[7] + b3p;
  V.p_rho0 = s_scl * s_scl * delta_v;
  V.p_h = (delta_v * s_scl) / P.v_scl;
  V.p_scl = P.table ? 1 / (V.p_h * P.step) : 1 / V.p_h;
  V.p_hs = 0.5 * (s_deg + 1) * V.p_h;
}

Params2D make_params2d(int fan, long nx, long ny, double s_scl, int s_deg, const double *cum_dev,
                       long size, double step, double coord0, long nv, double v_scl)
{
  Params2D P;
  std::memset(&P, 0, sizeof(P));
  P.nx = (int)nx;
  P.ny = (int)ny;
  P.nv = (int)nv;
  P.fan = fan;
  P.table = cum_dev ? 1 : 0;
  P.v_scl = v_scl;
  P.rho0_init = s_scl * s_scl;
  P.h_init = s_scl / v_scl;
  P.hs0 = 0.5 * (s_deg + 1);
  P.cum = cum_dev;
  P.last = (double)(size - 1);
  P.step = cum_dev ? step : 1.0;
  P.coord0 = coord0;
  return P;
}

// Per-view Long-Fessler constants (LongFessler2D.c:61-76).
LFView make_lfview(const trtt_b200_lf2d_parameters *p, double beta, double detector_offset)
{
  LFView g;
  std::memset(&g, 0, sizeof(g));
  g.cb = std::cos(beta);
  g.sb = std::sin(beta);
  const double off_y = g.cb * (p->objectOffset1) + g.sb * (p->objectOffset2);
  const double off_x = -g.sb * (p->objectOffset1) + g.cb * (p->objectOffset2);
  g.n1 = (int)p->objectDimension1;
  g.n2 = (int)p->objectDimension2;
  g.nd = (int)p->detectorDimension;
  g.vs = p->voxelSize;
  g.ps = p->pixelSize;
  g.sd = p->sourceDistance;
  g.x0 = off_x - 0.5 * (p->objectDimension1 - 1) * g.vs;
  g.y0 = off_y - 0.5 * (p->objectDimension2 - 1) * g.vs;
  g.off = detector_offset / p->pixelStep + 0.5 * (p->detectorDimension - 1);
  g.scale = (p->sourceDistance + p->detectorDistance) / p->pixelStep;
  g.size = p->pixelSize / p->pixelStep;
  return g;
}

bool lf_params_ok(const trtt_b200_lf2d_parameters *p)
{
  return p && dim_ok(p->objectDimension1) && dim_ok(p->objectDimension2) &&
         dim_ok(p->detectorDimension) &&
         p->objectDimension1 * p->objectDimension2 < (1L << 31);
}

int check_flag(DropIn &D, const char *what)
{
  int herr = 0;
  TRTT_CK(cudaMemcpyAsync(&herr, D.err.p, sizeof(int), cudaMemcpyDeviceToHost, D.stream));
  TRTT_CK(cudaStreamSynchronize(D.stream));
  if (herr & TRTT_ERR_SOURCE_PLANE) {
    std::fprintf(stderr, "trtt_b200 %s: a pixel lies on the source line (wk == 0); out left unchanged\n", what);
    return fail(std::string(what) + ": a pixel lies on the source line (wk == 0)");
  }
  if (herr) return fail(std::string(what) + ": device error flag set");
  return 0;
}

// out += H in (job 0) or H^T in (job != 0) on host arrays, one or more views.
int host2d(int fan, double *out, const double *in, long nx, long ny, double s_scl, int s_deg,
           const double *cum, long size, double step, const double *coord, long nv,
           double v_scl, long nviews, const double *xos, const double *xsd, int job,
           const char *what)
{
  clear_error();
  if (!out || !in || !xos || !xsd) return fail(std::string(what) + ": null array argument");
  if (!dim_ok(nx) || !dim_ok(ny) || !dim_ok(nv) || !dim_ok(nviews) || nx * ny >= (1L << 31))
    return fail(std::string(what) + ": dimensions out of range");
  if (cum && (size < 1 || !coord)) return fail(std::string(what) + ": invalid footprint table");
  if (nv * 4 > 200 * 1024) return fail(std::string(what) + ": detector too wide for one CTA");
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const long npix = nx * ny, ndet = nv * nviews;
  const long nin = job == 0 ? npix : ndet, nout = job == 0 ? ndet : npix;
  const double *cum_dev = nullptr;
  if (cum) {
    TRTT_CK(D.aux.ensure(sizeof(double) * size));
    TRTT_CK(cudaMemcpyAsync(D.aux.p, cum, sizeof(double) * size, cudaMemcpyHostToDevice, st));
    cum_dev = D.aux.as<double>();
  }
  Params2D P = make_params2d(fan, nx, ny, s_scl, s_deg, cum_dev, size, step, cum ? coord[0] : 0.0,
                             nv, v_scl);
  std::vector<View2D> hv(nviews);
  for (long v = 0; v < nviews; ++v) make_view2d(P, s_scl, s_deg, xos + 12 * v, xsd + 12 * v, hv[v]);
  TRTT_CK(D.geom.ensure(sizeof(View2D) * nviews));
  TRTT_CK(cudaMemcpyAsync(D.geom.p, hv.data(), sizeof(View2D) * nviews, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.err.ensure(sizeof(int)));
  TRTT_CK(cudaMemsetAsync(D.err.p, 0, sizeof(int), st));
  TRTT_CK(D.in64.ensure(sizeof(double) * nin));
  TRTT_CK(cudaMemcpyAsync(D.in64.p, in, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.vol32.ensure(sizeof(float) * nin));
  TRTT_CK(D.det32.ensure(sizeof(float) * nout));
  TRTT_CK(f64_to_f32(D.in64.as<double>(), D.vol32.as<float>(), nin, st));
  TRTT_CK(cudaMemsetAsync(D.det32.p, 0, sizeof(float) * nout, st));
  if (job == 0)
    TRTT_CK(launch_fwd2d(P, D.geom.as<View2D>(), (int)nviews, D.vol32.as<float>(),
                         D.det32.as<float>(), D.err.as<int>(), st));
  else
    TRTT_CK(launch_back2d(P, D.geom.as<View2D>(), (int)nviews, D.vol32.as<float>(),
                          D.det32.as<float>(), D.err.as<int>(), st));
  count_launch(3);
  if (check_flag(D, what)) return -1;
  TRTT_CK(D.out64.ensure(sizeof(double) * nout));
  TRTT_CK(cudaMemcpyAsync(D.out64.p, out, sizeof(double) * nout, cudaMemcpyHostToDevice, st));
  TRTT_CK(f32_add_to_f64(D.det32.as<float>(), D.out64.as<double>(), nout, st));
  count_launch();
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

int sparser2d(int fan, double *out, long i, long j, long nx, long ny, double s_scl, int s_deg,
              const double *cum, long size, double step, const double *coord, long nv,
              double v_scl, const double *xos, const double *xsd, const char *what)
{
  clear_error();
  if (!out || !cum || !coord || !xos || !xsd) return fail(std::string(what) + ": null argument");
  if (!dim_ok(nv) || size < 1) return fail(std::string(what) + ": dimensions out of range");
  if (i < -(1L << 30) || i > (1L << 30) || j < -(1L << 30) || j > (1L << 30))
    return fail(std::string(what) + ": pixel index out of range");
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  TRTT_CK(D.aux.ensure(sizeof(double) * size));
  TRTT_CK(cudaMemcpyAsync(D.aux.p, cum, sizeof(double) * size, cudaMemcpyHostToDevice, st));
  Params2D P = make_params2d(fan, nx > 0 ? nx : 1, ny > 0 ? ny : 1, s_scl, s_deg, D.aux.as<double>(),
                             size, step, coord[0], nv, v_scl);
  View2D hv;
  make_view2d(P, s_scl, s_deg, xos, xsd, hv);
  TRTT_CK(D.geom.ensure(sizeof(View2D)));
  TRTT_CK(cudaMemcpyAsync(D.geom.p, &hv, sizeof(View2D), cudaMemcpyHostToDevice, st));
  TRTT_CK(D.err.ensure(sizeof(int)));
  TRTT_CK(cudaMemsetAsync(D.err.p, 0, sizeof(int), st));
  TRTT_CK(D.out64.ensure(sizeof(double) * nv));
  TRTT_CK(cudaMemcpyAsync(D.out64.p, out, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
  TRTT_CK(launch_sparser2d(P, D.geom.as<View2D>(), (int)i, (int)j, D.out64.as<double>(),
                           D.err.as<int>(), st));
  count_launch();
  if (check_flag(D, what)) return -1;
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

// Long-Fessler host call: dst (= clr ? 0 : dst) += H src (direct) or H^T src.
void host_lf(const void *pv, double beta, double offset, const double *src, double *dst,
             int clr, int direct, int line, const char *what)
{
  clear_error();
  const trtt_b200_lf2d_parameters *p = static_cast<const trtt_b200_lf2d_parameters *>(pv);
  if (!lf_params_ok(p) || !src || !dst) {
    fail(std::string(what) + ": invalid arguments");
    return;
  }
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  cudaError_t e = D.init();
  if (e != cudaSuccess) {
    fail_cuda(e, what);
    return;
  }
  cudaSetDevice(D.device);
  cudaStream_t st = D.stream;
  const long npix = p->objectDimension1 * p->objectDimension2, nd = p->detectorDimension;
  const long nin = direct ? npix : nd, nout = direct ? nd : npix;
  if (nd * 4 > 200 * 1024) {
    fail(std::string(what) + ": detector too wide for one CTA");
    return;
  }
  LFView g = make_lfview(p, beta, offset);
#define LF_CK(call)                     \
  do {                                  \
    cudaError_t e_ = (call);            \
    if (e_ != cudaSuccess) {            \
      fail_cuda(e_, #call);             \
      return;                           \
    }                                   \
  } while (0)
  LF_CK(D.geom.ensure(sizeof(LFView)));
  LF_CK(cudaMemcpyAsync(D.geom.p, &g, sizeof(LFView), cudaMemcpyHostToDevice, st));
  LF_CK(D.in64.ensure(sizeof(double) * nin));
  LF_CK(cudaMemcpyAsync(D.in64.p, src, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
  LF_CK(D.vol32.ensure(sizeof(float) * nin));
  LF_CK(D.det32.ensure(sizeof(float) * nout));
  LF_CK(f64_to_f32(D.in64.as<double>(), D.vol32.as<float>(), nin, st));
  LF_CK(cudaMemsetAsync(D.det32.p, 0, sizeof(float) * nout, st));
  if (direct)
    LF_CK(launch_lf_fwd(D.geom.as<LFView>(), 1, (int)nd, line, D.vol32.as<float>(), D.det32.as<float>(), st));
  else
    LF_CK(launch_lf_back(D.geom.as<LFView>(), 1, (int)npix, line, D.vol32.as<float>(), D.det32.as<float>(), st));
  LF_CK(D.out64.ensure(sizeof(double) * nout));
  if (clr)
    LF_CK(cudaMemsetAsync(D.out64.p, 0, sizeof(double) * nout, st));
  else
    LF_CK(cudaMemcpyAsync(D.out64.p, dst, sizeof(double) * nout, cudaMemcpyHostToDevice, st));
  LF_CK(f32_add_to_f64(D.det32.as<float>(), D.out64.as<double>(), nout, st));
  count_launch(3);
  LF_CK(cudaMemcpyAsync(dst, D.out64.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, st));
  LF_CK(cudaStreamSynchronize(st));
}

void host_lf_sparser(const void *pv, double beta, double offset, long i1, long i2, double *dst,
                     int clr, int line, const char *what)
{
  clear_error();
  const trtt_b200_lf2d_parameters *p = static_cast<const trtt_b200_lf2d_parameters *>(pv);
  if (!lf_params_ok(p) || !dst) {
    fail(std::string(what) + ": invalid arguments");
    return;
  }
  if (i1 < -(1L << 30) || i1 > (1L << 30) || i2 < -(1L << 30) || i2 > (1L << 30)) {
    fail(std::string(what) + ": voxel index out of range");
    return;
  }
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  cudaError_t e = D.init();
  if (e != cudaSuccess) {
    fail_cuda(e, what);
    return;
  }
  cudaSetDevice(D.device);
  cudaStream_t st = D.stream;
  const long nd = p->detectorDimension;
  LFView g = make_lfview(p, beta, offset);
  LF_CK(D.geom.ensure(sizeof(LFView)));
  LF_CK(cudaMemcpyAsync(D.geom.p, &g, sizeof(LFView), cudaMemcpyHostToDevice, st));
  LF_CK(D.out64.ensure(sizeof(double) * nd));
  if (clr)
    LF_CK(cudaMemsetAsync(D.out64.p, 0, sizeof(double) * nd, st));
  else
    LF_CK(cudaMemcpyAsync(D.out64.p, dst, sizeof(double) * nd, cudaMemcpyHostToDevice, st));
  LF_CK(launch_lf_sparser(D.geom.as<LFView>(), line, (int)i1, (int)i2, D.out64.as<double>(), st));
  count_launch();
  LF_CK(cudaMemcpyAsync(dst, D.out64.p, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
  LF_CK(cudaStreamSynchronize(st));
#undef LF_CK
}

}  // namespace

extern "C" {

// ---- 2D B-spline projectors ----------------------------------------------
int trtt_PB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
              double *footprint, double *cum_footprint, long size_footprint,
              double step_footprint, double *coord_footprint, long nv, double v_scl,
              double *xos, double *xsd, int job)
{
  (void)footprint;
  if (!cum_footprint) return fail("trtt_PB2D: null cum_footprint");
  return host2d(0, out, in, nx, ny, s_scl, s_deg, cum_footprint, size_footprint, step_footprint,
                coord_footprint, nv, v_scl, 1, xos, xsd, job, "trtt_PB2D");
}

int trtt_FB2D(double *out, double *in, long nx, long ny, double s_scl, int s_deg,
              double *footprint, double *cum_footprint, long size_footprint,
              double step_footprint, double *coord_footprint, long nv, double v_scl,
              double *xos, double *xsd, int job)
{
  (void)footprint;
  if (!cum_footprint) return fail("trtt_FB2D: null cum_footprint");
  return host2d(1, out, in, nx, ny, s_scl, s_deg, cum_footprint, size_footprint, step_footprint,
                coord_footprint, nv, v_scl, 1, xos, xsd, job, "trtt_FB2D");
}

int trtt_PB2D_cubic(double *out, double *in, long nx, long ny, double s_scl, int s_deg, long nv,
                    double v_scl, double *xos, double *xsd, int job)
{
  return host2d(0, out, in, nx, ny, s_scl, s_deg, nullptr, 0, 1.0, nullptr, nv, v_scl, 1, xos,
                xsd, job, "trtt_PB2D_cubic");
}

int trtt_FB2D_cubic(double *out, double *in, long nx, long ny, double s_scl, int s_deg, long nv,
                    double v_scl, double *xos, double *xsd, int job)
{
  return host2d(1, out, in, nx, ny, s_scl, s_deg, nullptr, 0, 1.0, nullptr, nv, v_scl, 1, xos,
                xsd, job, "trtt_FB2D_cubic");
}

int trtt_PB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl, int s_deg,
                      double *footprint, double *cum_footprint, long size_footprint,
                      double step_footprint, double *coord_footprint, long nv, double v_scl,
                      double *xos, double *xsd)
{
  (void)footprint;
  return sparser2d(0, out, i, j, nx, ny, s_scl, s_deg, cum_footprint, size_footprint,
                   step_footprint, coord_footprint, nv, v_scl, xos, xsd, "trtt_PB2D_sparser");
}

int trtt_FB2D_sparser(double *out, long i, long j, long nx, long ny, double s_scl, int s_deg,
                      double *footprint, double *cum_footprint, long size_footprint,
                      double step_footprint, double *coord_footprint, long nv, double v_scl,
                      double *xos, double *xsd)
{
  (void)footprint;
  return sparser2d(1, out, i, j, nx, ny, s_scl, s_deg, cum_footprint, size_footprint,
                   step_footprint, coord_footprint, nv, v_scl, xos, xsd, "trtt_FB2D_sparser");
}

// ---- Long-Fessler -------------------------------------------------------
void lf2d_direct(const void *p, double beta, double detectorOffset, const double voxel[],
                 double pixel[], int clr)
{
  host_lf(p, beta, detectorOffset, voxel, pixel, clr, 1, 0, "lf2d_direct");
}

void lf2d_line_integ_direct(const void *p, double beta, double detectorOffset,
                            const double voxel[], double pixel[], int clr)
{
  host_lf(p, beta, detectorOffset, voxel, pixel, clr, 1, 1, "lf2d_line_integ_direct");
}

void lf2d_adjoint(const void *p, double beta, double detectorOffset, const double pixel[],
                  double voxel[], int clr)
{
  host_lf(p, beta, detectorOffset, pixel, voxel, clr, 0, 0, "lf2d_adjoint");
}

void lf2d_line_integ_adjoint(const void *p, double beta, double detectorOffset,
                             const double pixel[], double voxel[], int clr)
{
  host_lf(p, beta, detectorOffset, pixel, voxel, clr, 0, 1, "lf2d_line_integ_adjoint");
}

void lf2d_sparser(const void *p, double beta, double detectorOffset, long i1, long i2,
                  double pixel[], int clr)
{
  host_lf_sparser(p, beta, detectorOffset, i1, i2, pixel, clr, 0, "lf2d_sparser");
}

void lf2d_line_integ_sparser(const void *p, double beta, double detectorOffset, long i1, long i2,
                             double pixel[], int clr)
{
  host_lf_sparser(p, beta, detectorOffset, i1, i2, pixel, clr, 1, "lf2d_line_integ_sparser");
}

// ---- distance-driven 3D parallel beam -----------------------------------
int trtt_DD_PB3D(double *out, double *in, long nx, long ny, long nz, double s_scl, long nu,
                 long nv, double u_scl, double v_scl, double *xos, double *xsd, int job)
{
  clear_error();
  if (!out || !in || !xos || !xsd) return fail("trtt_DD_PB3D: null argument");
  if (!dim_ok(nx) || !dim_ok(ny) || !dim_ok(nz) || !dim_ok(nu) || !dim_ok(nv))
    return fail("trtt_DD_PB3D: dimensions out of range");
  // constants in the reference's order (plugin/trtt_3D_projectors.c:1081-1123)
  const double a1 = xsd[0], a2 = xsd[1], a3 = xsd[2], a4 = xsd[3];
  const double a5 = xsd[4], a6 = xsd[5], a7 = xsd[6], a8 = xsd[7];
  const double a9 = xsd[8], a10 = xsd[9], a11 = xsd[10], a12 = xsd[11];
  const double o5 = xos[4], o6 = xos[5], o7 = xos[6], o8 = xos[7];
  const double o9 = xos[8], o10 = xos[9], o11 = xos[10], o12 = xos[11];
  const double a1inv = -1.0 * (1.0 / a1);
  const double b1 = a6 + a1inv * a5 * a2, c1 = a10 + a1inv * a9 * a2;
  const double b2 = a7 + a1inv * a5 * a3, c2 = a11 + a1inv * a9 * a3;
  const double b3 = a8 + a1inv * a5 * a4, c3 = a12 + a1inv * a9 * a4;
  ParamsDD P;
  std::memset(&P, 0, sizeof(P));
  P.nx = (int)nx; P.ny = (int)ny; P.nz = (int)nz; P.nu = (int)nu; P.nv = (int)nv;
  P.u_scl = u_scl;
  P.v_scl = v_scl;
  P.v_x = b1 * o5 + b2 * o9;  P.u_x = c1 * o5 + c2 * o9;
  P.v_y = b1 * o6 + b2 * o10; P.u_y = c1 * o6 + c2 * o10;
  P.v_z = b1 * o7 + b2 * o11; P.u_z = c1 * o7 + c2 * o11;
  P.v_c = b1 * o8 + b2 * o12 + b3; P.u_c = c1 * o8 + c2 * o12 + c3;
  double Du = std::fabs(P.u_z);
  double Dv = (std::fabs(P.v_y) > std::fabs(P.v_x)) ? std::fabs(P.v_y) : std::fabs(P.v_x);
  P.h_norm = (s_scl * s_scl * s_scl) / (u_scl * v_scl * Du * Dv);
  P.Du = 0.5 * Du;
  P.Dv = 0.5 * Dv;
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const long nvox = nx * ny * nz, ndet = nu * nv;
  const long nin = job == 0 ? nvox : ndet, nout = job == 0 ? ndet : nvox;
  TRTT_CK(D.in64.ensure(sizeof(double) * nin));
  TRTT_CK(cudaMemcpyAsync(D.in64.p, in, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.out64.ensure(sizeof(double) * nout));
  TRTT_CK(cudaMemcpyAsync(D.out64.p, out, sizeof(double) * nout, cudaMemcpyHostToDevice, st));
  if (job == 0)
    TRTT_CK(launch_dd_fwd(P, D.in64.as<double>(), D.out64.as<double>(), st));
  else
    TRTT_CK(launch_dd_back(P, D.in64.as<double>(), D.out64.as<double>(), st));
  count_launch();
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

// ---- distance-driven 3D cone beam ---------------------------------------
// The reference's unfinished trtt_DD_CB3D (plugin/trtt_3D_projectors.c:
// 1340-1434, commented out there) completed as in the oracle; per-view
// coefficients in the reference's operand order.
static ParamsDDC ddc_view(long nx, long ny, long nz, double s_scl, long nu, long nv, double u_scl,
                          double v_scl, const double *xos, const double *xsd)
{
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
  ParamsDDC P;
  std::memset(&P, 0, sizeof(P));
  P.nx = (int)nx; P.ny = (int)ny; P.nz = (int)nz; P.nu = (int)nu; P.nv = (int)nv;
  P.u_scl = u_scl;
  P.v_scl = v_scl;
  P.s3 = s_scl * s_scl * s_scl;
  P.o1 = o1; P.o2 = o2; P.o3 = o3; P.o4 = o4;
  P.nv_x = b1 * o5 + b2 * o9;  P.nu_x = c1 * o5 + c2 * o9;
  P.nv_y = b1 * o6 + b2 * o10; P.nu_y = c1 * o6 + c2 * o10;
  P.nv_z = b1 * o7 + b2 * o11; P.nu_z = c1 * o7 + c2 * o11;
  P.nv_c = b1 * o8 + b2 * o12; P.nu_c = c1 * o8 + c2 * o12;
  P.d_x = a1 * o1 + a2 * o5 + a3 * o9;
  P.d_y = a1 * o2 + a2 * o6 + a3 * o10;
  P.d_z = a1 * o3 + a2 * o7 + a3 * o11;
  P.d_c = a1 * o4 + a2 * o8 + a3 * o12;
  P.a4sqr = a4 * a4;
  P.a4m = -1.0 * a4;
  P.a8 = a8;
  P.a12 = a12;
  P.b3 = b3;
  P.c3 = c3;
  P.axis = (std::fabs(P.nv_y) > std::fabs(P.nv_x)) ? 2 : 1;
  return P;
}

int trtt_b200_dd_cb3d(double *out, const double *in, long nx, long ny, long nz, double s_scl,
                      long nu, long nv, double u_scl, double v_scl, long nviews, const double *xos,
                      const double *xsd, int job)
{
  clear_error();
  if (!out || !in || !xos || !xsd) return fail("dd_cb3d: null argument");
  if (!dim_ok(nx) || !dim_ok(ny) || !dim_ok(nz) || !dim_ok(nu) || !dim_ok(nv) || nviews < 1 ||
      nviews > 65535)
    return fail("dd_cb3d: dimensions out of range (views in [1, 65535])");
  std::vector<ParamsDDC> hv(nviews);
  for (long v = 0; v < nviews; ++v)
    hv[v] = ddc_view(nx, ny, nz, s_scl, nu, nv, u_scl, v_scl, xos + 12 * v, xsd + 12 * v);
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const long nvox = nx * ny * nz, ndet = nu * nv * nviews;
  const long nin = job == 0 ? nvox : ndet, nout = job == 0 ? ndet : nvox;
  TRTT_CK(D.geom.ensure(sizeof(ParamsDDC) * nviews));
  TRTT_CK(cudaMemcpyAsync(D.geom.p, hv.data(), sizeof(ParamsDDC) * nviews, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.err.ensure(sizeof(int)));
  TRTT_CK(cudaMemsetAsync(D.err.p, 0, sizeof(int), st));
  TRTT_CK(D.in64.ensure(sizeof(double) * nin));
  TRTT_CK(cudaMemcpyAsync(D.in64.p, in, sizeof(double) * nin, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.out64.ensure(sizeof(double) * nout));
  TRTT_CK(cudaMemcpyAsync(D.out64.p, out, sizeof(double) * nout, cudaMemcpyHostToDevice, st));
  const ParamsDDC *vd = static_cast<const ParamsDDC *>(D.geom.p);
  if (job == 0)
    TRTT_CK(launch_ddc_fwd(vd, (int)nviews, nvox, D.in64.as<double>(), D.out64.as<double>(), nu * nv,
                           D.err.as<int>(), st));
  else
    TRTT_CK(launch_ddc_back(vd, (int)nviews, nvox, D.in64.as<double>(), nu * nv, D.out64.as<double>(),
                            D.err.as<int>(), st));
  count_launch();
  int herr = 0;
  TRTT_CK(cudaMemcpyAsync(&herr, D.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  if (herr) {
    std::fprintf(stderr, "trtt_b200: a voxel lies in the source plane (wk == 0); out left unchanged\n");
    return fail("dd_cb3d: a voxel lies in the source plane (wk == 0)");
  }
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * nout, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

int trtt_DD_CB3D(double *out, double *in, long nx, long ny, long nz, double s_scl, long nu,
                 long nv, double u_scl, double v_scl, double *xos, double *xsd, int job)
{
  return trtt_b200_dd_cb3d(out, in, nx, ny, nz, s_scl, nu, nv, u_scl, v_scl, 1, xos, xsd, job);
}

// ---- 1-based COO product ------------------------------------------------
int trtt_mvmult(double *out, double *in, long number, double *a, long *i, long *j)
{
  clear_error();
  if (number < 0) return fail("trtt_mvmult: negative number of coefficients");
  if (number == 0) return 0;
  if (!out || !in || !a || !i || !j) return fail("trtt_mvmult: null argument");
  // the reference ABI carries no array lengths: the extents are the largest
  // indices used; indices below 1 are rejected (the reference would write
  // before the start of the array)
  long imax = 0, jmax = 0;
  for (long k = 0; k < number; ++k) {
    if (i[k] < 1 || j[k] < 1) return fail("trtt_mvmult: index below 1 (indices are 1-based)");
    if (i[k] > imax) imax = i[k];
    if (j[k] > jmax) jmax = j[k];
  }
  DropIn &D = dropin();
  std::lock_guard<std::mutex> lock(D.mu);
  TRTT_CK(D.init());
  TRTT_CK(cudaSetDevice(D.device));
  cudaStream_t st = D.stream;
  const size_t bytes_idx = sizeof(long) * number;
  TRTT_CK(D.aux.ensure(sizeof(double) * number + 2 * bytes_idx + 64));
  double *a_d = D.aux.as<double>();
  long *i_d = reinterpret_cast<long *>(D.aux.as<char>() + sizeof(double) * number);
  long *j_d = reinterpret_cast<long *>(D.aux.as<char>() + sizeof(double) * number + bytes_idx);
  TRTT_CK(cudaMemcpyAsync(a_d, a, sizeof(double) * number, cudaMemcpyHostToDevice, st));
  TRTT_CK(cudaMemcpyAsync(i_d, i, bytes_idx, cudaMemcpyHostToDevice, st));
  TRTT_CK(cudaMemcpyAsync(j_d, j, bytes_idx, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.in64.ensure(sizeof(double) * jmax));
  TRTT_CK(cudaMemcpyAsync(D.in64.p, in, sizeof(double) * jmax, cudaMemcpyHostToDevice, st));
  TRTT_CK(D.out64.ensure(sizeof(double) * imax));
  TRTT_CK(cudaMemcpyAsync(D.out64.p, out, sizeof(double) * imax, cudaMemcpyHostToDevice, st));
  TRTT_CK(launch_mvmult(a_d, i_d, j_d, number, D.in64.as<double>(), D.out64.as<double>(), st));
  count_launch();
  TRTT_CK(cudaMemcpyAsync(out, D.out64.p, sizeof(double) * imax, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Native 2D plan (device float*, all views in one launch)
// ---------------------------------------------------------------------------
struct trtt_b200_plan2d {
  int lf = 0;          // 0: B-spline projector, 1: Long-Fessler
  int line = 0;        // Long-Fessler line-integral variant
  long nviews = 0, npix = 0, ndet = 0;
  Params2D P;
  DevBuf views, cum, err;
};

extern "C" int trtt_b200_plan2d_create(trtt_b200_plan2d **plan, int geometry, long nx, long ny,
                                       double s_scl, int s_deg, const double *cum_footprint,
                                       long size_footprint, double step_footprint,
                                       const double *coord_footprint, long nv, double v_scl,
                                       long nviews, const double *xos, const double *xsd)
{
  clear_error();
  if (!plan) return fail("plan2d_create: null plan pointer");
  *plan = nullptr;
  if (geometry != TRTT_B200_PARALLEL_BEAM && geometry != TRTT_B200_FAN_BEAM &&
      geometry != TRTT_B200_CONE_BEAM)
    return fail("plan2d_create: geometry must be 3 (parallel) or 5 (fan)");
  if (!dim_ok(nx) || !dim_ok(ny) || !dim_ok(nv) || !dim_ok(nviews) || nx * ny >= (1L << 31))
    return fail("plan2d_create: dimensions out of range");
  if (nv * 4 > 200 * 1024) return fail("plan2d_create: detector too wide for one CTA");
  if (!xos || !xsd) return fail("plan2d_create: null xos/xsd");
  if (cum_footprint && (size_footprint < 1 || !coord_footprint))
    return fail("plan2d_create: invalid footprint table");
  trtt_b200_plan2d *pl = new (std::nothrow) trtt_b200_plan2d();
  if (!pl) return fail("plan2d_create: out of host memory");
  cudaError_t e = cudaSuccess;
  if (cum_footprint) {
    e = pl->cum.ensure(sizeof(double) * size_footprint);
    if (e == cudaSuccess)
      e = cudaMemcpy(pl->cum.p, cum_footprint, sizeof(double) * size_footprint, cudaMemcpyHostToDevice);
  }
  pl->P = make_params2d(geometry != TRTT_B200_PARALLEL_BEAM, nx, ny, s_scl, s_deg,
                        cum_footprint ? pl->cum.as<double>() : nullptr, size_footprint,
                        step_footprint, cum_footprint ? coord_footprint[0] : 0.0, nv, v_scl);
  std::vector<View2D> hv(nviews);
  for (long v = 0; v < nviews; ++v) make_view2d(pl->P, s_scl, s_deg, xos + 12 * v, xsd + 12 * v, hv[v]);
  if (e == cudaSuccess) e = pl->views.ensure(sizeof(View2D) * nviews);
  if (e == cudaSuccess)
    e = cudaMemcpy(pl->views.p, hv.data(), sizeof(View2D) * nviews, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = pl->err.ensure(sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(pl->err.p, 0, sizeof(int));
  if (e != cudaSuccess) {
    delete pl;
    return fail_cuda(e, "plan2d_create");
  }
  pl->nviews = nviews;
  pl->npix = nx * ny;
  pl->ndet = nv;
  *plan = pl;
  return 0;
}

extern "C" int trtt_b200_plan2d_create_lf(trtt_b200_plan2d **plan, const void *params,
                                          int line_integ, long nviews, const double *beta,
                                          const double *offset)
{
  clear_error();
  if (!plan) return fail("plan2d_create_lf: null plan pointer");
  *plan = nullptr;
  const trtt_b200_lf2d_parameters *p = static_cast<const trtt_b200_lf2d_parameters *>(params);
  if (!lf_params_ok(p) || !dim_ok(nviews) || !beta || !offset)
    return fail("plan2d_create_lf: invalid arguments");
  if (p->detectorDimension * 4 > 200 * 1024) return fail("plan2d_create_lf: detector too wide");
  trtt_b200_plan2d *pl = new (std::nothrow) trtt_b200_plan2d();
  if (!pl) return fail("plan2d_create_lf: out of host memory");
  pl->lf = 1;
  pl->line = line_integ ? 1 : 0;
  std::vector<LFView> hv(nviews);
  for (long v = 0; v < nviews; ++v) hv[v] = make_lfview(p, beta[v], offset[v]);
  cudaError_t e = pl->views.ensure(sizeof(LFView) * nviews);
  if (e == cudaSuccess)
    e = cudaMemcpy(pl->views.p, hv.data(), sizeof(LFView) * nviews, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = pl->err.ensure(sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(pl->err.p, 0, sizeof(int));
  if (e != cudaSuccess) {
    delete pl;
    return fail_cuda(e, "plan2d_create_lf");
  }
  pl->nviews = nviews;
  pl->npix = p->objectDimension1 * p->objectDimension2;
  pl->ndet = p->detectorDimension;
  *plan = pl;
  return 0;
}

extern "C" int trtt_b200_plan2d_forward(trtt_b200_plan2d *pl, const float *img, float *sino,
                                        void *stream)
{
  clear_error();
  if (!pl || !img || !sino) return fail("plan2d_forward: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (pl->lf)
    TRTT_CK(launch_lf_fwd(pl->views.as<LFView>(), (int)pl->nviews, (int)pl->ndet, pl->line, img, sino, st));
  else
    TRTT_CK(launch_fwd2d(pl->P, pl->views.as<View2D>(), (int)pl->nviews, img, sino, pl->err.as<int>(), st));
  count_launch();
  return 0;
}

extern "C" int trtt_b200_plan2d_backward(trtt_b200_plan2d *pl, const float *sino, float *img,
                                         void *stream)
{
  clear_error();
  if (!pl || !img || !sino) return fail("plan2d_backward: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (pl->lf)
    TRTT_CK(launch_lf_back(pl->views.as<LFView>(), (int)pl->nviews, (int)pl->npix, pl->line, sino, img, st));
  else
    TRTT_CK(launch_back2d(pl->P, pl->views.as<View2D>(), (int)pl->nviews, sino, img, pl->err.as<int>(), st));
  count_launch();
  return 0;
}

extern "C" int trtt_b200_plan2d_status(trtt_b200_plan2d *pl, void *stream)
{
  clear_error();
  if (!pl) return fail("plan2d_status: null plan");
  int h = 0;
  TRTT_CK(cudaStreamSynchronize((cudaStream_t)stream));
  TRTT_CK(cudaMemcpy(&h, pl->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  TRTT_CK(cudaMemset(pl->err.p, 0, sizeof(int)));
  if (h & TRTT_ERR_SOURCE_PLANE) return fail("a pixel lies on the source line (wk == 0)");
  if (h) return fail("device error flag set");
  return 0;
}

extern "C" int trtt_b200_plan2d_destroy(trtt_b200_plan2d *pl)
{
  if (!pl) return 0;
  pl->views.release();
  pl->cum.release();
  pl->err.release();
  delete pl;
  return 0;
}

// Per-view COO assembly of a 2D B-spline system matrix on the GPU (replaces
// the temp-file builder of Ytrtt_2D_projectors.i:212-369): slot
// s = (view*npix + p)*max_cells + l holds (a, row, col) for footprint cell l
// of pixel p, 1-based rows (detector cell) and columns (pixel); unused slots
// have row = col = 0.  a/rows/cols are device arrays of nviews*npix*max_cells.
extern "C" int trtt_b200_plan2d_assemble(trtt_b200_plan2d *pl, int max_cells, double *a,
                                         long *rows, long *cols, void *stream)
{
  clear_error();
  if (!pl || !a || !rows || !cols) return fail("plan2d_assemble: null argument");
  if (pl->lf) return fail("plan2d_assemble: B-spline plans only");
  if (max_cells < 1 || max_cells > 4096) return fail("plan2d_assemble: max_cells out of range");
  cudaStream_t st = (cudaStream_t)stream;
  const long per = pl->npix * (long)max_cells;
  for (long v = 0; v < pl->nviews; ++v) {
    TRTT_CK(launch_assemble2d(pl->P, pl->views.as<View2D>() + v, 1, max_cells, a + v * per,
                              rows + v * per, cols + v * per, pl->err.as<int>(), st));
    count_launch();
  }
  return 0;
}
