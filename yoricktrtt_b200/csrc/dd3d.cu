// dd3d.cu -- distance-driven 3D parallel-beam projector (trtt_DD_PB3D,
// plugin/trtt_3D_projectors.c:1077-1173, footprints :406-526 and :817-944)
// and the 1-based COO sparse product of trtt_mvmult
// (plugin/trtt_common.c:62-69).
//
// DD: each voxel projects to an axis-aligned rectangle whose per-cell
// overlap lengths are computed in FP64 exactly as the reference computes
// them, including the transpose's v-axis fill in which every fully covered
// cell writes the same slot (plugin/trtt_3D_projectors.c:903-917); the
// direct projector scatters with FP64 atomics, the transpose gathers per
// voxel.
#include <cuda_runtime.h>

#include "kernels2d.h"
#include "trtt_device.cuh"

namespace trtt {

struct DDAxis {
  double b1, b2, up, down, left, scl;
  long nint;  // (long)(down - up): < 0 when both bounds fall in one cell
  long neff;  // (long)(ceil(b2) - left): number of cells touched
};

__device__ __forceinline__ void dd_axis(double c, double D, int n, double scl, DDAxis &a)
{
  const double last = (double)(n - 1);
  double b1 = dsub(c, D), b2 = dadd(c, D);
  b1 = b1 >= 0 ? b1 : 0;
  b1 = b1 <= last ? b1 : last;
  b2 = b2 >= 0 ? b2 : 0;
  b2 = b2 <= last ? b2 : last;
  a.b1 = b1;
  a.b2 = b2;
  a.up = ceil(b1);
  a.down = floor(b2);
  a.left = floor(b1);
  a.scl = scl;
  a.nint = (long)dsub(a.down, a.up);
  a.neff = (long)dsub(ceil(b2), a.left);
}

// Overlap length of cell l of the axis (plugin/trtt_3D_projectors.c:443-475).
// `broken` reproduces the transpose's v fill (single-slot writes).
__device__ __forceinline__ double dd_cell(const DDAxis &a, long l, bool broken)
{
  if (a.nint < 0) return l == 0 ? dmul(a.scl, dsub(a.b2, a.b1)) : 0.0;
  const long off = (a.up > a.b1) ? 1 : 0;
  if (off && l == 0) return dmul(a.scl, dsub(a.up, a.b1));
  if (!broken) {
    const long idx = l - off;
    if (idx < a.nint) return a.scl;
    if (idx == a.nint && a.down < a.b2) return dmul(a.scl, dsub(a.b2, a.down));
    return 0.0;
  }
  if (l != off) return 0.0;
  if (a.down < a.b2) return dmul(a.scl, dsub(a.b2, a.down));
  return a.nint > 0 ? a.scl : 0.0;
}

__device__ __forceinline__ void dd_voxel(const ParamsDD &P, long idx, DDAxis &au, DDAxis &av,
                                         long &base)
{
  const int i = (int)(idx % P.nx);
  const long r = idx / P.nx;
  const int j = (int)(r % P.ny);
  const int k = (int)(r / P.ny);
  const double di = i, dj = j, dk = k;
  const double vc = dadd(dadd(dadd(dmul(P.v_z, dk), P.v_c), dmul(P.v_y, dj)), dmul(P.v_x, di));
  const double uc = dadd(dadd(dadd(dmul(P.u_z, dk), P.u_c), dmul(P.u_y, dj)), dmul(P.u_x, di));
  dd_axis(uc, P.Du, P.nu, P.u_scl, au);
  dd_axis(vc, P.Dv, P.nv, P.v_scl, av);
  base = (long)av.left * P.nu + (long)au.left;
}

__global__ void k_dd_fwd(const ParamsDD P, const double *__restrict__ vol, double *__restrict__ det)
{
  const long n = (long)P.nx * P.ny * P.nz;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const double x = vol[idx];
  DDAxis au, av;
  long base;
  dd_voxel(P, idx, au, av, base);
  if (!(au.neff > 0 && av.neff > 0)) return;
  for (long m = 0; m < av.neff; ++m) {
    const double hv = dmul(P.h_norm, dd_cell(av, m, false));
    for (long l = 0; l < au.neff; ++l)
      atomicAdd(det + base + m * P.nu + l, dmul(dmul(hv, dd_cell(au, l, false)), x));
  }
}

__global__ void k_dd_back(const ParamsDD P, const double *__restrict__ det, double *__restrict__ vol)
{
  const long n = (long)P.nx * P.ny * P.nz;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  DDAxis au, av;
  long base;
  dd_voxel(P, idx, au, av, base);
  if (!(au.neff > 0 && av.neff > 0)) return;
  double acc = vol[idx];
  for (long m = 0; m < av.neff; ++m) {
    const double hv = dmul(P.h_norm, dd_cell(av, m, true));
    for (long l = 0; l < au.neff; ++l)
      acc = dadd(acc, dmul(dmul(hv, dd_cell(au, l, false)), det[base + m * P.nu + l]));
  }
  vol[idx] = acc;
}

cudaError_t launch_dd_fwd(const ParamsDD &P, const double *vol, double *det, cudaStream_t st)
{
  const long n = (long)P.nx * P.ny * P.nz;
  k_dd_fwd<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, vol, det);
  return cudaGetLastError();
}

cudaError_t launch_dd_back(const ParamsDD &P, const double *det, double *vol, cudaStream_t st)
{
  const long n = (long)P.nx * P.ny * P.nz;
  k_dd_back<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, det, vol);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// 1-based COO product: out[i[k]-1] += a[k] * in[j[k]-1]
// ---------------------------------------------------------------------------
__global__ void k_mvmult(const double *__restrict__ a, const long *__restrict__ i,
                         const long *__restrict__ j, long nnz, const double *__restrict__ in,
                         double *__restrict__ out)
{
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (long)gridDim.x * blockDim.x) {
    const double v = dmul(a[k], in[j[k] - 1]);
    if (v != 0.0) atomicAdd(out + (i[k] - 1), v);
  }
}

cudaError_t launch_mvmult(const double *a, const long *i, const long *j, long nnz,
                          const double *in, double *out, cudaStream_t st)
{
  if (nnz <= 0) return cudaSuccess;
  long g = (nnz + 255) / 256;
  if (g > 148L * 32) g = 148L * 32;
  k_mvmult<<<(unsigned)g, 256, 0, st>>>(a, i, j, nnz, in, out);
  return cudaGetLastError();
}

}  // namespace trtt
