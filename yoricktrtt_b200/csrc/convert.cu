// convert.cu -- volume layout and precision conversions.
//
// The reference stores a volume as [k][j][i] (x fastest,
// plugin/trtt_common.h:248).  The projector kernels walk voxel columns
// along k, so they keep volumes as [j][i][k] (k fastest): a column is one
// contiguous, coalesced run.  Viewing the XYZ volume as an (nz x ncols)
// matrix, the conversion is a transpose; it is done through 32x33 shared
// tiles so both the read and the write are coalesced.
#include <cuda_runtime.h>

#include "kernels.h"

namespace trtt {

template <typename Tin, typename Tout, bool ADD>
__global__ void __launch_bounds__(256)
k_transpose(const Tin *__restrict__ src, Tout *__restrict__ dst, long rows,
            long cols, long batch_stride)
{
  // src is rows x cols (row-major), dst is cols x rows (row-major)
  __shared__ float tile[32][33];
  const long b = blockIdx.z;
  src += b * batch_stride;
  dst += b * batch_stride;
  const long c0 = (long)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const long rtiles = (rows + 31) / 32;
  for (long rt = blockIdx.y; rt < rtiles; rt += gridDim.y) {
    const long r0 = rt * 32;
    for (int y = ty; y < 32; y += 8) {
      const long r = r0 + y, c = c0 + tx;
      if (r < rows && c < cols) tile[y][tx] = (float)src[r * cols + c];
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
      const long c = c0 + y, r = r0 + tx;
      if (r < rows && c < cols) {
        if (ADD) dst[c * rows + r] += (Tout)tile[tx][y];
        else dst[c * rows + r] = (Tout)tile[tx][y];
      }
    }
    __syncthreads();
  }
}

template <typename Tin, typename Tout, bool ADD>
static cudaError_t transpose(const Tin *src, Tout *dst, long rows, long cols,
                             int nb, cudaStream_t st)
{
  if (rows <= 0 || cols <= 0 || nb <= 0) return cudaSuccess;
  long rt = (rows + 31) / 32;
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)(rt < 65535 ? rt : 65535), nb);
  k_transpose<Tin, Tout, ADD><<<grid, 256, 0, st>>>(src, dst, rows, cols, rows * cols);
  return cudaGetLastError();
}

cudaError_t xyz_f64_to_col_f32(const double *src, float *dst, int nx, int ny,
                               int nz, int nb, cudaStream_t st)
{
  return transpose<double, float, false>(src, dst, nz, (long)nx * ny, nb, st);
}

cudaError_t xyz_f32_to_col_f32(const float *src, float *dst, int nx, int ny,
                               int nz, int nb, cudaStream_t st)
{
  return transpose<float, float, false>(src, dst, nz, (long)nx * ny, nb, st);
}

cudaError_t col_f32_add_to_xyz_f64(const float *src, double *dst, int nx,
                                   int ny, int nz, int nb, cudaStream_t st)
{
  return transpose<float, double, true>(src, dst, (long)nx * ny, nz, nb, st);
}

cudaError_t col_f32_add_to_xyz_f32(const float *src, float *dst, int nx,
                                   int ny, int nz, int nb, cudaStream_t st)
{
  return transpose<float, float, true>(src, dst, (long)nx * ny, nz, nb, st);
}

__global__ void k_f64_to_f32(const double *__restrict__ s, float *__restrict__ d, long n)
{
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    d[t] = (float)s[t];
}

__global__ void k_f32_add_to_f64(const float *__restrict__ s, double *__restrict__ d, long n)
{
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    d[t] += (double)s[t];
}

static unsigned grid_for(long n)
{
  long g = (n + 255) / 256;
  if (g > 148L * 16) g = 148L * 16;
  return (unsigned)(g > 0 ? g : 1);
}

cudaError_t f64_to_f32(const double *src, float *dst, long n, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_f64_to_f32<<<grid_for(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

cudaError_t f32_add_to_f64(const float *src, double *dst, long n, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_f32_add_to_f64<<<grid_for(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace trtt
