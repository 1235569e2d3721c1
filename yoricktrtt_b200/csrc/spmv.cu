// spmv.cu -- FP64 product of a CSR sparse matrix with a vector, the
// precomputed-matrix mode of the 2D projectors.
//
// The reference can precompute each view's system matrix from the sparsers
// (Ytrtt_2D_projectors.i:212-369, yeti sparse_matrix) and then evaluates
// H x and H^T y by sparse products (Tomography_2D/Ytrtt2D_optim.i:320-387,
// trtt_mvmult, plugin/trtt_common.c:62-69).  On the GPU the matrix comes from
// trtt_b200_plan2d_assemble (COO slots grouped by pixel); the caller sorts
// it into compressed rows (for H and for H^T) once, and every product is one
// launch of k_csr_spmv: one warp per row, lanes strided over the row's
// entries (coalesced column and value reads), FP64 products summed by a warp
// reduction, no atomics.  A column index outside [0, ncols) is skipped and
// recorded in a flag read by trtt_b200_csr_status.
#include <cuda_runtime.h>

#include "runtime.h"
#include "trtt_b200.h"

namespace trtt {
namespace {

__device__ int g_csr_bad_index;

__global__ void k_csr_spmv(const long *__restrict__ row_ptr, const long *__restrict__ col,
                           const double *__restrict__ val, long nrows, long ncols,
                           const double *__restrict__ x, double *__restrict__ y, int accumulate)
{
  const long row = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const long b = row_ptr[row], e = row_ptr[row + 1];
  double acc = 0.0;
  for (long k = b + lane; k < e; k += 32) {
    const long c = col[k];
    if (c < 0 || c >= ncols) {
      atomicOr(&g_csr_bad_index, 1);
      continue;
    }
    acc += val[k] * x[c];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) y[row] = accumulate ? y[row] + acc : acc;
}

}  // namespace
}  // namespace trtt

extern "C" int trtt_b200_csr_spmv(const long *row_ptr, const long *col, const double *val, long nrows,
                                  long ncols, const double *x, double *y, int accumulate, void *stream)
{
  using namespace trtt;
  clear_error();
  if (nrows < 0 || ncols < 0) return fail("csr_spmv: negative dimension");
  if (nrows == 0) return 0;
  if (!row_ptr || !x || !y || ((!col || !val) && ncols > 0)) return fail("csr_spmv: null argument");
  const long threads = nrows * 32;
  const long blocks = (threads + 255) / 256;
  if (blocks > 0x7fffffffL) return fail("csr_spmv: too many rows");
  k_csr_spmv<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(row_ptr, col, val, nrows, ncols, x, y,
                                                                   accumulate);
  TRTT_CK(cudaGetLastError());
  count_launch();
  return 0;
}

extern "C" int trtt_b200_csr_status(void *stream)
{
  using namespace trtt;
  clear_error();
  TRTT_CK(cudaStreamSynchronize((cudaStream_t)stream));
  int h = 0;
  TRTT_CK(cudaMemcpyFromSymbol(&h, g_csr_bad_index, sizeof(int)));
  if (h) {
    const int z = 0;
    TRTT_CK(cudaMemcpyToSymbol(g_csr_bad_index, &z, sizeof(int)));
    return fail("csr_spmv: a column index was out of range (entry skipped)");
  }
  return 0;
}
