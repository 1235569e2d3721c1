// proj2d.cu -- 2D B-spline projectors (trtt_PB2D/FB2D, table and closed-form
// cubic; plugin/trtt_2D_projectors.c:186-536,
// plugin/trtt_2D_projectors_cubic.c:209-398) and the Long-Fessler
// separable-footprint fan-beam model
// (tomography-LongFessler-model/LongFessler2D.c:41-681).
//
// 2D problems are small (a 512^2 image has 0.26 M pixels), so all geometry
// is evaluated in FP64 with the reference's operation order (no fused
// multiply-add); only the accumulations are FP32 (direct, shared-memory
// detector row) or FP64 (transpose, per pixel in registers).
//
// Direct: one CTA per view owns the view's detector row in shared memory
// and scatters every pixel's footprint into it; the row is written back
// once.  Transpose: one thread per pixel gathers over all views.
#include <cuda_runtime.h>

#include "kernels2d.h"
#include "trtt_device.cuh"

namespace trtt {

// ---------------------------------------------------------------------------
// B-spline 2D: per-pixel footprint
// ---------------------------------------------------------------------------
struct Foot2D {
  int lo, n;
  double start, inc;
  double rho0;
};

// Footprint of pixel (i,j) for view V.  Returns -1 if the pixel lies on the
// source line (fan beam, wk == 0), 0 otherwise (n may be 0).
__device__ __forceinline__ int foot2d(const Params2D &P, const View2D &V, int i, int j,
                                      Foot2D &f)
{
  const double di = (double)i, dj = (double)j;
  double vc, h, scl, hs;
  if (P.fan) {
    // plugin/trtt_2D_projectors.c:330-352
    double wk = dadd(dadd(dmul(V.o2, dj), V.o4), dmul(V.o1, di));
    double num = dadd(dadd(dmul(V.b1o6, dj), V.b1o8), dmul(V.b1o5, di));
    double den = dadd(dadd(dmul(V.d_y, dj), V.d_c), dmul(V.d_x, di));
    vc = dadd(dmul(ddiv(V.a4m, den), num), V.b3);
    if (wk == 0.0) {
      f.n = 0;
      return -1;
    }
    double magn = ddiv(V.a4m, wk);
    double vca8 = dmul(dsub(vc, V.a8), P.v_scl);
    double delta_v = dsqrt(dadd(1.0, ddiv(dmul(vca8, vca8), V.a4sqr)));
    f.rho0 = dmul(dmul(P.rho0_init, magn), delta_v);
    h = dmul(dmul(P.h_init, magn), delta_v);
    scl = P.table ? ddiv(1.0, dmul(h, P.step)) : ddiv(1.0, h);
    hs = dmul(P.hs0, h);
  } else {
    // plugin/trtt_2D_projectors.c:222-226
    vc = dadd(dadd(dmul(V.b1o6, dj), V.b1o8b3), dmul(V.b1o5, di));
    f.rho0 = V.p_rho0;
    h = V.p_h;
    scl = V.p_scl;
    hs = V.p_hs;
  }
  if (!isfinite(vc)) {
    f.n = 0;
    return 0;
  }
  const int lo = clamp_left_cell(dsub(vc, hs), P.nv);
  const int hi = clamp_right_cell(dadd(vc, hs), P.table ? P.nv - 1 : P.nv - 2);
  f.lo = lo;
  f.n = hi - lo;
  if (P.table) {
    // (vl - (vc + coord0*h)) * scl   (plugin/trtt_2D_projectors.c:94-97)
    f.start = dmul(dsub((double)lo, dadd(vc, dmul(P.coord0, h))), scl);
  } else {
    // (vl - vc) * scl   (plugin/trtt_2D_projectors_cubic.c:119)
    f.start = dmul(dsub((double)lo, vc), scl);
  }
  f.inc = scl;
  return 0;
}

// Primitive at edge l of a 2D footprint (exact FP64, reference order).
__device__ __forceinline__ double edge2d(const Params2D &P, const Foot2D &f, int l)
{
  const double x = (l == 0) ? f.start : dadd(f.start, dmul((double)l, f.inc));
  if (P.table) return __ldg(P.cum + table_slot(x, P.last));
  return cubic_prim_d(x);
}

__global__ void __launch_bounds__(1024)
k_fwd2d(const Params2D P, const View2D *__restrict__ views,
        const float *__restrict__ img, float *__restrict__ sino, int *__restrict__ err)
{
  extern __shared__ float acc[];
  const View2D V = views[blockIdx.x];
  for (int t = threadIdx.x; t < P.nv; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  const int npix = P.nx * P.ny;
  for (int p = threadIdx.x; p < npix; p += blockDim.x) {
    const float x = __ldg(img + p);
    if (x == 0.0f) continue;
    const int i = p % P.nx, j = p / P.nx;
    Foot2D f;
    if (foot2d(P, V, i, j, f)) {
      atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      continue;
    }
    if (f.n <= 0) continue;
    const double xr = (double)x * f.rho0;
    double p0 = edge2d(P, f, 0);
    for (int l = 0; l < f.n; ++l) {
      double p1 = edge2d(P, f, l + 1);
      atomicAdd(acc + f.lo + l, (float)((p1 - p0) * xr));
      p0 = p1;
    }
  }
  __syncthreads();
  float *out = sino + (long)blockIdx.x * P.nv;
  for (int t = threadIdx.x; t < P.nv; t += blockDim.x) out[t] += acc[t];
}

__global__ void __launch_bounds__(256)
k_back2d(const Params2D P, const View2D *__restrict__ views, int nviews,
         const float *__restrict__ sino, float *__restrict__ img, int *__restrict__ err)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nx * P.ny) return;
  const int i = p % P.nx, j = p / P.nx;
  double acc = 0.0;
  for (int v = 0; v < nviews; ++v) {
    Foot2D f;
    if (foot2d(P, views[v], i, j, f)) {
      atomicOr(err, TRTT_ERR_SOURCE_PLANE);
      continue;
    }
    if (f.n <= 0) continue;
    const float *row = sino + (long)v * P.nv + f.lo;
    double s = 0.0;
    double p0 = edge2d(P, f, 0);
    for (int l = 0; l < f.n; ++l) {
      double p1 = edge2d(P, f, l + 1);
      s = fma(p1 - p0, (double)__ldg(row + l), s);
      p0 = p1;
    }
    acc = fma(f.rho0, s, acc);
  }
  img[p] += (float)acc;
}

// Column (i,j) of the 2D system matrix: out[v] += w(v) (sparser).
__global__ void k_sparser2d(const Params2D P, const View2D *__restrict__ views,
                            int i, int j, double *__restrict__ out, int *__restrict__ err)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Foot2D f;
  if (foot2d(P, views[0], i, j, f)) {
    atomicOr(err, TRTT_ERR_SOURCE_PLANE);
    return;
  }
  double p0 = edge2d(P, f, 0);
  for (int l = 0; l < f.n; ++l) {
    double p1 = edge2d(P, f, l + 1);
    // table: rho0*vox*(diff); cubic: (diff*vox)*rho0 with vox = 1
    out[f.lo + l] += P.table ? f.rho0 * (p1 - p0) : (p1 - p0) * f.rho0;
    p0 = p1;
  }
}

// Sparse assembly of one view's system matrix: for every pixel p the
// footprint cells and weights, as 1-based COO triplets (row = detector
// cell, column = pixel index + 1).  Slot s = p * max_cells + l; unused slots
// get row = 0.
__global__ void k_assemble2d(const Params2D P, const View2D *__restrict__ views,
                             int max_cells, double *__restrict__ a, long *__restrict__ rows,
                             long *__restrict__ cols, int *__restrict__ err)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nx * P.ny) return;
  const int i = p % P.nx, j = p / P.nx;
  const long base = (long)p * max_cells;
  Foot2D f;
  int n = 0;
  if (foot2d(P, views[blockIdx.y], i, j, f)) {
    atomicOr(err, TRTT_ERR_SOURCE_PLANE);
  } else {
    n = f.n > 0 ? f.n : 0;
    if (n > max_cells) {
      atomicOr(err, TRTT_ERR_BAD_INDEX);
      n = max_cells;
    }
    double p0 = n ? edge2d(P, f, 0) : 0.0;
    for (int l = 0; l < n; ++l) {
      double p1 = edge2d(P, f, l + 1);
      a[base + l] = P.table ? f.rho0 * (p1 - p0) : (p1 - p0) * f.rho0;
      rows[base + l] = f.lo + l + 1;
      cols[base + l] = p + 1;
      p0 = p1;
    }
  }
  for (int l = n; l < max_cells; ++l) {
    a[base + l] = 0.0;
    rows[base + l] = 0;
    cols[base + l] = 0;
  }
}

// ---------------------------------------------------------------------------
// Long-Fessler separable footprint (LongFessler2D.c:90-139)
// ---------------------------------------------------------------------------
struct LFVoxel {
  double t[4];
  double obliq;
  int kf, kl;
};

__device__ __forceinline__ void lf_voxel(const LFView &g, int i1, int i2, LFVoxel &o)
{
  const double y = dadd(g.y0, dmul((double)i2, g.vs));
  const double y1 = dsub(y, dmul(0.5, g.vs)), y2 = dadd(y, dmul(0.5, g.vs));
  const double x = dadd(g.x0, dmul((double)i1, g.vs));
  const double x1 = dsub(x, dmul(0.5, g.vs)), x2 = dadd(x, dmul(0.5, g.vs));
  auto S = [&](double X, double Y) {
    double numr = dmul(g.scale, dadd(dmul(Y, g.sb), dmul(X, g.cb)));
    double denr = dsub(g.sd, dsub(dmul(Y, g.cb), dmul(X, g.sb)));
    return dadd(ddiv(numr, denr), g.off);
  };
  double t0 = S(x1, y1), t1 = S(x2, y1), t2 = S(x1, y2), t3 = S(x2, y2), tmp;
#define LF_SWAP(a, b) if (a > b) { tmp = a; a = b; b = tmp; }
  LF_SWAP(t0, t1);
  LF_SWAP(t2, t3);
  LF_SWAP(t0, t2);
  LF_SWAP(t1, t3);
  LF_SWAP(t1, t2);
#undef LF_SWAP
  o.t[0] = t0; o.t[1] = t1; o.t[2] = t2; o.t[3] = t3;
  const double qx = dadd(x, dmul(g.sd, g.sb));
  const double qy = dsub(y, dmul(g.sd, g.cb));
  const double q = (fabs(qy) > fabs(qx)) ? ddiv(qx, qy) : ddiv(qy, qx);
  o.obliq = dsqrt(dadd(1.0, dmul(q, q)));
  long kf = (long)floor(dsub(t0, dmul(0.5, g.size)));
  if (kf < 0) kf = 0;
  long kl = (long)ceil(dadd(t3, dmul(0.5, g.size)));
  if (kl >= g.nd) kl = g.nd - 1;
  o.kf = (int)(kf > (long)g.nd ? g.nd : kf);
  o.kl = (int)(kl < -1 ? -1 : kl);
}

__device__ __forceinline__ double lf_tri(double a, double b, double c)
{
  if (a >= b) return 0.0;
  return ddiv(dmul(dadd(b, a), dsub(b, a)), dadd(c, c));
}
__device__ __forceinline__ double lf_rect(double a, double b)
{
  if (a >= b) return 0.0;
  return dsub(b, a);
}
__device__ __forceinline__ double lf_max(double a, double b) { return a >= b ? a : b; }
__device__ __forceinline__ double lf_min(double a, double b) { return a <= b ? a : b; }

// Cell weight: trapezoid integral over cell k (LongFessler2D.c:129-136) or
// trapezoid height at its centre (line-integral variant, :226-234).
__device__ __forceinline__ double lf_cell(const LFVoxel &o, int k, double size, int line)
{
  const double *t = o.t;
  const double dk = (double)k;
  if (line) {
    if (dk >= t[0] && dk < t[1]) return ddiv(dsub(dk, t[0]), dsub(t[1], t[0]));
    if (dk >= t[1] && dk < t[2]) return 1.0;
    if (dk >= t[2] && dk < t[3]) return ddiv(dsub(dk, t[3]), dsub(t[2], t[3]));
    return 0.0;
  }
  const double s1 = dsub(dk, dmul(0.5, size));
  const double s2 = dadd(s1, size);
  return dadd(dadd(lf_tri(dsub(lf_max(s1, t[0]), t[0]), dsub(lf_min(s2, t[1]), t[0]), dsub(t[1], t[0])),
                   lf_rect(lf_max(s1, t[1]), lf_min(s2, t[2]))),
              lf_tri(dsub(t[3], lf_min(s2, t[3])), dsub(t[3], lf_max(s1, t[2])), dsub(t[3], t[2])));
}

__global__ void __launch_bounds__(1024)
k_lf_fwd(const LFView *__restrict__ views, int line, const float *__restrict__ img,
         float *__restrict__ sino)
{
  extern __shared__ float acc[];
  const LFView g = views[blockIdx.x];
  for (int t = threadIdx.x; t < g.nd; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  const int npix = g.n1 * g.n2;
  const double alpha0 = line ? g.vs : dmul(g.vs, g.ps);
  for (int p = threadIdx.x; p < npix; p += blockDim.x) {
    const float x = __ldg(img + p);
    if (x == 0.0f) continue;
    LFVoxel o;
    lf_voxel(g, p % g.n1, p / g.n1, o);
    const double alpha = dmul(dmul(o.obliq, alpha0), (double)x);
    for (int k = o.kf; k <= o.kl; ++k) {
      const double w = lf_cell(o, k, g.size, line);
      if (w != 0.0) atomicAdd(acc + k, (float)(w * alpha));
    }
  }
  __syncthreads();
  float *out = sino + (long)blockIdx.x * g.nd;
  for (int t = threadIdx.x; t < g.nd; t += blockDim.x) out[t] += acc[t];
}

__global__ void __launch_bounds__(256)
k_lf_back(const LFView *__restrict__ views, int nviews, int line,
          const float *__restrict__ sino, float *__restrict__ img)
{
  const LFView &g0 = views[0];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g0.n1 * g0.n2) return;
  const int i1 = p % g0.n1, i2 = p / g0.n1;
  double acc = 0.0;
  for (int v = 0; v < nviews; ++v) {
    const LFView &g = views[v];
    LFVoxel o;
    lf_voxel(g, i1, i2, o);
    const double alpha = line ? dmul(o.obliq, g.vs) : dmul(o.obliq, dmul(g.vs, g.ps));
    const float *row = sino + (long)v * g.nd;
    double s = 0.0;
    for (int k = o.kf; k <= o.kl; ++k)
      s = fma(dmul(alpha, lf_cell(o, k, g.size, line)), (double)__ldg(row + k), s);
    acc += s;
  }
  img[p] += (float)acc;
}

__global__ void k_lf_sparser(const LFView *__restrict__ views, int line, int i1, int i2,
                             double *__restrict__ out)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const LFView &g = views[0];
  LFVoxel o;
  lf_voxel(g, i1, i2, o);
  const double alpha = line ? dmul(o.obliq, g.vs) : dmul(o.obliq, dmul(g.vs, g.ps));
  for (int k = o.kf; k <= o.kl; ++k) {
    if (line) {
      // (alpha*(k-t0))/(t1-t0) etc. (LongFessler2D.c:663-671)
      const double *t = o.t;
      const double dk = (double)k;
      if (dk >= t[0] && dk < t[1]) out[k] += ddiv(dmul(alpha, dsub(dk, t[0])), dsub(t[1], t[0]));
      else if (dk >= t[1] && dk < t[2]) out[k] += alpha;
      else if (dk >= t[2] && dk < t[3]) out[k] += ddiv(dmul(alpha, dsub(dk, t[3])), dsub(t[2], t[3]));
    } else {
      out[k] += dmul(lf_cell(o, k, g.size, 0), alpha);
    }
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
cudaError_t launch_fwd2d(const Params2D &P, const View2D *views, int nviews, const float *img,
                         float *sino, int *err, cudaStream_t st)
{
  k_fwd2d<<<nviews, 1024, sizeof(float) * P.nv, st>>>(P, views, img, sino, err);
  return cudaGetLastError();
}

cudaError_t launch_back2d(const Params2D &P, const View2D *views, int nviews, const float *sino,
                          float *img, int *err, cudaStream_t st)
{
  const int npix = P.nx * P.ny;
  k_back2d<<<(npix + 255) / 256, 256, 0, st>>>(P, views, nviews, sino, img, err);
  return cudaGetLastError();
}

cudaError_t launch_sparser2d(const Params2D &P, const View2D *view, int i, int j, double *out,
                             int *err, cudaStream_t st)
{
  k_sparser2d<<<1, 32, 0, st>>>(P, view, i, j, out, err);
  return cudaGetLastError();
}

cudaError_t launch_assemble2d(const Params2D &P, const View2D *views, int nviews, int max_cells,
                              double *a, long *rows, long *cols, int *err, cudaStream_t st)
{
  const int npix = P.nx * P.ny;
  dim3 grid((npix + 255) / 256, nviews);
  k_assemble2d<<<grid, 256, 0, st>>>(P, views, max_cells, a, rows, cols, err);
  return cudaGetLastError();
}

cudaError_t launch_lf_fwd(const LFView *views, int nviews, int nd, int line, const float *img,
                          float *sino, cudaStream_t st)
{
  k_lf_fwd<<<nviews, 1024, sizeof(float) * nd, st>>>(views, line, img, sino);
  return cudaGetLastError();
}

cudaError_t launch_lf_back(const LFView *views, int nviews, int npix, int line, const float *sino,
                           float *img, cudaStream_t st)
{
  k_lf_back<<<(npix + 255) / 256, 256, 0, st>>>(views, nviews, line, sino, img);
  return cudaGetLastError();
}

cudaError_t launch_lf_sparser(const LFView *view, int line, int i1, int i2, double *out,
                              cudaStream_t st)
{
  k_lf_sparser<<<1, 32, 0, st>>>(view, line, i1, i2, out);
  return cudaGetLastError();
}

}  // namespace trtt
