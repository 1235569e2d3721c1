// persist4d.cu -- the weighted least-squares data term of a (4D) scan in
// one persistent launch:
//
//   resid = W (H x - y),  cost = 1/2 sum W (H x - y)^2,  grad += H^T resid
//
// with H the gate-interpolated cone/parallel-beam projector of every view
// (view k sees w0 x[g0] + w1 x[g1]; the transpose adds w_j H_k^T r_k into
// gate j), which is the cost evaluation of the 4D reconstruction
// (Tomography_4D/Ytrtt4D_optim.i:87-223; per-gate projection
// Ytrtt_3D_projectors.i:254-375).  Closed-form (cubic) model, column-
// factorised views.
//
// One cooperative launch of as many CTAs as fit on the GPU pulls work items
// from a device queue:
//   items [0, nb):        band items (view, detector-row band): the direct
//                         projection of the band in shared memory, written
//                         back as the weighted residual with the band's
//                         FP64 cost;
//   items [nb, nb + nc):  column items (block of columns, k range): the
//                         transpose gathered from the residuals, each view
//                         once, into the view's two gates (with one gate, or
//                         gates too many for shared memory: one item per
//                         gate, block of columns and k range, over the
//                         gate's views).
// The uneven view counts of the gates need no padding: the queue holds
// exactly one item per band and per column block.  A column item needs
// every band item finished; a CTA that draws one waits on the count of
// finished band items.  All band items have been drawn by then and every
// CTA is resident (cooperative launch), so the wait ends -- but it is
// bounded all the same (%globaltimer): past the limit the CTA sets
// TRTT_ERR_STALL in the error word and returns.  The CTA that finishes
// the last band item sums the band costs in item order (deterministic).
#include <cuda_runtime.h>

#include <algorithm>

#include "fast3d_items.cuh"
#include "kernels.h"

namespace trtt {

namespace {

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int GEOM, int KP, int MINB>
__global__ void __launch_bounds__(512, MINB)
k_wls_persistent(const WlsLaunch A)
{
  extern __shared__ float sm[];
  __shared__ View3D sV;
  __shared__ int s_next, s_item, s_ok;
  __shared__ double s_red[16];
  const Params3D &P = A.P;
  const int nwarps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv;
  const int R = A.band_rows;
  const int nb = A.n_band_items, nc = A.n_col_items;
  const int ncols = P.nx * P.ny;
  const int colblocks = (ncols + nwarps - 1) / nwarps;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(A.queue, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= nb + nc) break;
    if (item < nb) {
      // ---- band item: residual and cost of rows [v0, v1) of one view ----
      const int vi = item / A.nbands, band = item - vi * A.nbands;
      const int v0 = band * R, v1 = min(v0 + R, nv);
      float *acc = sm;
      float *prof = sm + R * nu + warp * nu;
      float *wv = sm + R * nu + nwarps * nu + warp * R;
      int *locks = reinterpret_cast<int *>(sm + R * nu + nwarps * nu + nwarps * R);
      if (threadIdx.x < (int)(sizeof(View3D) / 8))
        reinterpret_cast<double *>(&sV)[threadIdx.x] =
            reinterpret_cast<const double *>(A.views + vi)[threadIdx.x];
      if (threadIdx.x == 0) s_next = 0;
      for (int t = threadIdx.x; t < R * nu; t += blockDim.x) acc[t] = 0.f;
      for (int t = threadIdx.x; t < R; t += blockDim.x) locks[t] = 0;
      for (int t = lane; t < nu; t += 32) prof[t] = 0.f;
      __syncthreads();
      band_item<GEOM>(P, sV, A.vol, A.gate_stride, v0, v1, R, acc, prof, wv, locks, &s_next, A.err,
                      A.lock_spread != 0);
      __syncthreads();
      const long off = (long)vi * nu * nv + (long)v0 * nu;
      const int ncell = (v1 - v0) * nu;
      double c = 0.0;
      for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
        const float r = acc[t] - __ldg(A.y + off + t);
        const float wr = A.w ? __ldg(A.w + off + t) * r : r;
        A.resid[off + t] = wr;
        c += (double)wr * (double)r;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULLM, c, o);
      if (lane == 0) s_red[warp] = c;
      __threadfence();  // this thread's residual stores, before the count
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < nwarps; ++q) t += s_red[q];
        A.cost_parts[item] = 0.5 * t;
        __threadfence();
        const unsigned done = atomicAdd(A.queue + 1, 1u) + 1u;
        s_ok = (done == (unsigned)nb) ? 1 : 0;
      }
      __syncthreads();
      if (s_ok && warp == 0) {
        // the last band item: total cost in item order
        __threadfence();
        double t = 0.0;
        for (int q = lane; q < nb; q += 32) t += __ldcg(A.cost_parts + q);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULLM, t, o);
        if (lane == 0) *A.cost = t;
      }
      __syncthreads();
    } else {
      // ---- column item: wait for every band item, then gather ----
      if (threadIdx.x == 0) {
        const unsigned need = (unsigned)nb + (unsigned)A.extra_wait;
        const unsigned long long t0 = global_ns();
        int ok = 1;
        while (*reinterpret_cast<volatile unsigned *>(A.queue + 1) < need) {
          if (global_ns() - t0 > (unsigned long long)A.wait_ns) {
            atomicOr(A.err, TRTT_ERR_STALL);
            ok = 0;
            break;
          }
          __nanosleep(200);
        }
        __threadfence();
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) break;
      const int ci = item - nb;
      if (A.gates_mode) {
        const int cb = ci / A.kchunks, kc = ci - cb * A.kchunks;
        const int col = cb * nwarps + warp;
        float *row = sm + (size_t)warp * back_gates_row(nu, A.ngates, KP);
        float *sacc = row + ((nu + 3) & ~3), *scmp = sacc + A.ngates * 64 * KP;
        if (col < ncols)
          column_item_gates<GEOM, KP, LoadCG>(P, A.views, A.pairs, 0, A.nviews, A.resid, (long)nu * nv,
                                              A.grad, A.gate_stride, A.ngates, col, kc * (64 * KP), row,
                                              sacc, scmp, A.err, (nu & 3) == 0);
      } else {
        const int per_gate = colblocks * A.kchunks;
        const int gate = ci / per_gate;
        const int rem = ci - gate * per_gate;
        const int cb = rem / A.kchunks, kc = rem - cb * A.kchunks;
        const int col = cb * nwarps + warp;
        if (col < ncols)
          column_item<GEOM, KP, LoadCG>(P, A.views, A.entries, A.gate_ptr[gate], A.gate_ptr[gate + 1],
                                        0, A.nviews, A.resid, (long)nu * nv, A.grad, A.gate_stride,
                                        col, kc * (64 * KP), gate, sm + warp * nu, A.err,
                                        (nu & 3) == 0);
      }
      __syncthreads();
    }
  }
}

template <int GEOM, int KP, int MINB>
cudaError_t launch_wls(WlsLaunch L, int sms, cudaStream_t st)
{
  auto kern = k_wls_persistent<GEOM, KP, MINB>;
  const size_t smem = std::max(wls_smem(L.P.nu, L.band_rows), wls_gates_smem(L.P.nu, L.ngates, KP, L.gates_mode));
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm > MINB) per_sm = MINB;
  const int grid = sms * per_sm;
  void *args[] = {&L};
  return cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(512), args, smem, st);
}

}  // namespace

size_t wls_smem(int nu, int band_rows)
{
  // band item: band + one profile and one weight row per warp (16 warps) +
  // one lock per row; column items use 16 * nu of it
  return sizeof(float) * ((size_t)band_rows * nu + 16 * (size_t)nu + 16 * (size_t)band_rows +
                          (size_t)band_rows);
}

// Shared memory of the column items over all gates: one profile row and
// the per-gate sums of every warp (16 warps); 0 when not in that mode.
size_t wls_gates_smem(int nu, int ngates, int kp, int gates_mode)
{
  return gates_mode ? sizeof(float) * 16 * back_gates_row(nu, ngates, kp) : 0;
}

int wls_kp(int nz)
{
  return nz <= 64 ? 1 : (nz <= 128 ? 2 : 4);
}

cudaError_t launch_wls_persistent(WlsLaunch L, int sms, cudaStream_t st)
{
  const int kp = wls_kp(L.P.nz);
  L.kchunks = (L.P.nz + 64 * kp - 1) / (64 * kp);
  L.nbands = (L.P.nv + L.band_rows - 1) / L.band_rows;
  L.n_band_items = L.nviews * L.nbands;
  L.lock_spread = band_lock_spread(L.P) ? 1 : 0;
  L.gates_mode = (L.pairs && L.ngates > 1 && wls_gates_smem(L.P.nu, L.ngates, kp, 1) <= 200u * 1024u) ? 1 : 0;
  L.n_col_items = (L.gates_mode ? 1 : L.ngates) * ((L.P.nx * L.P.ny + 15) / 16) * L.kchunks;
  const bool cone = L.P.geom == GEOM_CONE;
  // CTAs per SM: 1 (up to 128 registers per thread) or 2 (64)
  const bool two = L.ctas_per_sm == 2;
#define TRTT_WLS_CASE(K)                                                                  \
  if (kp == K) {                                                                          \
    if (two) return cone ? launch_wls<GEOM_CONE, K, 2>(L, sms, st) : launch_wls<GEOM_PARALLEL, K, 2>(L, sms, st); \
    return cone ? launch_wls<GEOM_CONE, K, 1>(L, sms, st) : launch_wls<GEOM_PARALLEL, K, 1>(L, sms, st);          \
  }
  TRTT_WLS_CASE(1)
  TRTT_WLS_CASE(2)
  TRTT_WLS_CASE(4)
#undef TRTT_WLS_CASE
  return cudaErrorInvalidValue;
}

}  // namespace trtt
