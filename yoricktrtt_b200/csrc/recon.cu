// recon.cu -- device kernels of the reconstruction layer around the
// projector pair: weighted residual with an FP64 cost, isotropic total
// variation (value in FP64 + gradient), cubic B-spline sampling of the
// coefficients and its adjoint, and FP64-accumulated inner products.
//
// Cost of the data term (Tomography_3D/Ytrtt3D_optim.i:186-201):
//   f = 1/2 sum_k (H_k x - y_k)' W_k (H_k x - y_k),  residual r = W (Hx - y)
// Regulariser (Tomography_3D/Ytrtt3D_optim.i:204-234): total variation of the
// voxel samples z = S x of the B-spline coefficients x (S: separable
// convolution with the cubic B-spline sampled at the integers,
// [1/6, 2/3, 1/6]; zero outside the object), gradient S' dTV/dz.  The
// reference delegates both to packages that are not in its repository
// (YTotVar, SPL); this is the standard smoothed isotropic form
// TV(z) = sum_i sqrt(|grad z|_i^2 + eps^2) with forward differences.
#include <cuda_runtime.h>

#include "runtime.h"
#include "trtt_b200.h"

namespace {

// Block-wide FP64 sum, added into *out (one atomic per block).
__device__ __forceinline__ void block_sum_add(double v, double *out)
{
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(out, v);
  }
}

__global__ void k_wls(const float *__restrict__ hx, const float *__restrict__ y,
                      const float *__restrict__ w, float *__restrict__ wr, long n,
                      double *__restrict__ f)
{
  double acc = 0.0;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const float r = hx[t] - y[t];
    const float wt = w ? w[t] : 1.0f;
    const float q = wt * r;
    wr[t] = q;
    acc += 0.5 * (double)q * (double)r;
  }
  block_sum_add(acc, f);
}

__global__ void k_dot(const float *__restrict__ a, const float *__restrict__ b, long n,
                      double *__restrict__ out)
{
  double acc = 0.0;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    acc += (double)a[t] * (double)b[t];
  block_sum_add(acc, out);
}

// Isotropic TV with forward differences, layout [k][j][i] (nz = 1 for 2D).
// Cell t contributes s_t = sqrt(dx^2 + dy^2 + dz^2 + eps^2) - eps; the
// gradient at sample t gathers the derivative of its own cell and of the
// three cells behind it (i-1, j-1, k-1), so every sample is written by one
// thread: g += mu * dTV/dz, f += mu * TV(z).
__device__ __forceinline__ void tv_cell(const float *__restrict__ z, long t, int i, int j, int k,
                                        int nx, int ny, int nz, float eps, float &dx, float &dy,
                                        float &dz, float &s)
{
  const float c = z[t];
  dx = (i + 1 < nx) ? z[t + 1] - c : 0.f;
  dy = (j + 1 < ny) ? z[t + nx] - c : 0.f;
  dz = (k + 1 < nz) ? z[t + (long)nx * ny] - c : 0.f;
  s = sqrtf(dx * dx + dy * dy + dz * dz + eps * eps);
}

__global__ void k_tv(const float *__restrict__ z, int nx, int ny, int nz, float eps, float mu,
                     float *__restrict__ g, double *__restrict__ f)
{
  const long n = (long)nx * ny * nz;
  const long sxy = (long)nx * ny;
  double acc = 0.0;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const long r = t / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    float dx, dy, dz, s;
    tv_cell(z, t, i, j, k, nx, ny, nz, eps, dx, dy, dz, s);
    acc += (double)s - (double)eps;
    float gv = -(dx + dy + dz) / s;
    if (i > 0) {
      float ax, ay, az, as;
      tv_cell(z, t - 1, i - 1, j, k, nx, ny, nz, eps, ax, ay, az, as);
      gv += ax / as;
    }
    if (j > 0) {
      float ax, ay, az, as;
      tv_cell(z, t - nx, i, j - 1, k, nx, ny, nz, eps, ax, ay, az, as);
      gv += ay / as;
    }
    if (k > 0) {
      float ax, ay, az, as;
      tv_cell(z, t - sxy, i, j, k - 1, nx, ny, nz, eps, ax, ay, az, as);
      gv += az / as;
    }
    g[t] += mu * gv;
  }
  block_sum_add(acc * (double)mu, f);
}

// One axis of the separable B-spline sampling [1/6, 2/3, 1/6] (symmetric, so
// the adjoint is the same convolution with zero boundaries).
__global__ void k_spline_axis(const float *__restrict__ src, float *__restrict__ dst, int nx,
                              int ny, int nz, int axis)
{
  const long n = (long)nx * ny * nz;
  const long stride = axis == 0 ? 1 : (axis == 1 ? nx : (long)nx * ny);
  const int len = axis == 0 ? nx : (axis == 1 ? ny : nz);
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int p = axis == 0 ? (int)(t % nx) : (axis == 1 ? (int)((t / nx) % ny) : (int)(t / ((long)nx * ny)));
    float v = (2.0f / 3.0f) * src[t];
    if (p > 0) v += (1.0f / 6.0f) * src[t - stride];
    if (p + 1 < len) v += (1.0f / 6.0f) * src[t + stride];
    dst[t] = v;
  }
}

unsigned grid_of(long n)
{
  long g = (n + 255) / 256;
  if (g > 148L * 8) g = 148L * 8;
  return (unsigned)(g > 0 ? g : 1);
}

}  // namespace

extern "C" {

int trtt_b200_wls_residual(const float *hx, const float *y, const float *w, float *wr, long n,
                           double *f_dev, void *stream)
{
  trtt::clear_error();
  if (!hx || !y || !wr || !f_dev || n < 0) return trtt::fail("wls_residual: invalid argument");
  if (n == 0) return 0;
  k_wls<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(hx, y, w, wr, n, f_dev);
  trtt::count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_dot(const float *a, const float *b, long n, double *out_dev, void *stream)
{
  trtt::clear_error();
  if (!a || !b || !out_dev || n < 0) return trtt::fail("dot: invalid argument");
  if (n == 0) return 0;
  k_dot<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(a, b, n, out_dev);
  trtt::count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_tv(const float *z, long nx, long ny, long nz, double eps, double mu, float *g,
                 double *f_dev, void *stream)
{
  trtt::clear_error();
  if (!z || !g || !f_dev || !trtt::dim_ok(nx) || !trtt::dim_ok(ny) || !trtt::dim_ok(nz) || !(eps > 0))
    return trtt::fail("tv: invalid argument");
  const long n = nx * ny * nz;
  k_tv<<<grid_of(n), 256, 0, (cudaStream_t)stream>>>(z, (int)nx, (int)ny, (int)nz, (float)eps,
                                                     (float)mu, g, f_dev);
  trtt::count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_spline_sample(const float *x, float *z, float *tmp, long nx, long ny, long nz,
                            void *stream)
{
  trtt::clear_error();
  if (!x || !z || !tmp || !trtt::dim_ok(nx) || !trtt::dim_ok(ny) || !trtt::dim_ok(nz))
    return trtt::fail("spline_sample: invalid argument");
  const long n = nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  k_spline_axis<<<grid_of(n), 256, 0, st>>>(x, z, (int)nx, (int)ny, (int)nz, 0);
  k_spline_axis<<<grid_of(n), 256, 0, st>>>(z, tmp, (int)nx, (int)ny, (int)nz, 1);
  if (nz > 1) {
    k_spline_axis<<<grid_of(n), 256, 0, st>>>(tmp, z, (int)nx, (int)ny, (int)nz, 2);
    trtt::count_launch(3);
  } else {
    TRTT_CK(cudaMemcpyAsync(z, tmp, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    trtt::count_launch(2);
  }
  TRTT_CK(cudaGetLastError());
  return 0;
}

}  // extern "C"
