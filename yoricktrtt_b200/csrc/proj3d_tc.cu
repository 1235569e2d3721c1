// proj3d_tc.cu -- direct 3D projector (closed-form cubic model, column-
// factorised views) whose band accumulation runs on the tensor cores.
//
// For a band of R detector rows of one view the direct projection is
//   out[r][u] = sum over columns c of  wv_c(r) * P_c(u),
// P_c the column's u-profile (sum over its voxels of rho * x * u-weight) and
// wv_c its v-weights on the band rows: the product of a (u x columns) and a
// (columns x rows) matrix.  Producer warps build P_c exactly as the CUDA-core
// band kernel does (column_profile) and write P_c and wv_c into K-slots of a
// shared-memory ring; one issuer thread multiplies complete groups of 4
// columns into an FP32 accumulator in tensor memory (tcgen05.mma kind::tf32,
// M = 128 cells of u, N = R rows, K = 8).  TF32 keeps 11 significant bits, so
// each value x is split into x_hi = TF32(x) and x_lo = TF32(x - x_hi), and a
// column takes four K entries: A = (P_hi, P_lo, P_hi, P_lo) against
// B = (w_hi, w_hi, w_lo, w_lo), whose dot product is (P_hi + P_lo) *
// (w_hi + w_lo) = P w to within 2^-21 relative.  One MMA (K = 8) covers two
// columns.  The shared-memory atomics of the CUDA-core spread (one per band
// row and cell of every column) become one 16-byte store per cell.
//
// Accuracy: each product is exact to FP32, but the accumulation into the
// FP32 tensor-memory accumulator rounds toward zero, so the error grows with
// the number of columns that reach a detector cell: at 256^3 -> 512^2
// (about 240 non-zero additions per cell) the band is 1.5-1.8e-5 (relative
// L2) from FP64, where the CUDA-core kernels stay below 1e-6.  The kernel is
// therefore an explicit option (set_tiles(TRTT_B200_TILES_TENSOR)), never
// the default; it meets 1e-5 on small scans only.
//
// Operand layout: the no-swizzle K-major canonical layout, 16 bytes = the 4
// K entries of one column, 8 rows (cells or band rows) of 16 bytes per core
// matrix: entry (m, column c, e) at (m/8)*SBO + c*128 + (m%8)*16 + e*4 bytes,
// LBO = 128 (core matrices adjacent in K), SBO = 4 columns * 128.  A warp
// storing one column (32 consecutive m, 16 bytes each) fills 4 whole
// 128-byte lines: no bank conflicts.
//
// Waits are bounded (2 s, %globaltimer).  On expiry the kernel sets
// TRTT_ERR_STALL, stops producing and issuing, waits (bounded) for the
// products it issued, frees its tensor memory and leaves the band unwritten.
#include <cuda_runtime.h>

#include "fast3d.cuh"
#include "kernels.h"
#include "tc100.cuh"

namespace trtt {
namespace {

constexpr int TC_PROD = 15;                // producer warps; warp TC_PROD issues
constexpr int TC_THREADS = 32 * (TC_PROD + 1);
constexpr int TC_G = 4;                    // columns per ring group (K = 4 * TC_G)
constexpr int TC_LBO = 128;                // bytes between K-adjacent core matrices
constexpr int TC_SBO = TC_G * 128;         // bytes between 8-row groups
constexpr uint64_t TC_LIMIT_NS = 2000000000ull;
constexpr int TC_SMEM_SM = 233472;         // shared memory of one SM (228 KB)
constexpr int TC_STATIC = 2048;            // static shared memory + the 1 KB per-CTA reserve, upper bound

struct TcShape {
  int rows = 0;    // band rows R = N of the MMA (multiple of 16), 0: unsupported
  int nuc = 0;     // 128-cell chunks of u
  int ng = 0;      // ring depth in groups of TC_G columns
  int tmem_cols = 0;
  int a_bytes = 0; // A operand of one group (nuc * 128 cells x TC_G columns x 16 bytes)
  int b_bytes = 0; // B operand of one group (rows x TC_G columns x 16 bytes)
  int prof_floats = 0;
  size_t smem = 0;
};

TcShape tc_shape(int nu)
{
  TcShape t;
  t.nuc = (nu + 127) / 128;
  if (t.nuc < 1 || t.nuc > 16) return TcShape{};
  int rows = 256 / t.nuc;
  rows -= rows % 16;
  if (rows > 64) rows = 64;
  t.rows = rows;
  int tc = 32;
  while (tc < t.nuc * rows) tc <<= 1;
  t.tmem_cols = tc;
  t.a_bytes = t.nuc * 16 * TC_SBO;
  t.b_bytes = rows / 8 * TC_SBO;
  t.prof_floats = (nu + 3) & ~3;
  const size_t fixed = sizeof(float) * (size_t)TC_PROD * t.prof_floats;
  for (int ng = 2; ng >= 1; --ng) {
    const size_t s = (size_t)ng * (t.a_bytes + t.b_bytes) + fixed;
    const bool two = 2 * (s + TC_STATIC) <= (size_t)TC_SMEM_SM;  // two CTAs per SM
    if (two || (ng == 1 && s + TC_STATIC <= (size_t)TC_SMEM_SM)) {
      t.ng = ng;
      t.smem = s;
      return t;
    }
  }
  return TcShape{};
}

__device__ __forceinline__ float tf32_rna(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// D[tmem] (+)= A * B^T, TF32 operands, FP32 accumulator, one thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
  const uint32_t z = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z),
        "r"(z)
      : "memory");
}

// Instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3, M >> 4.
__host__ __device__ constexpr uint32_t idesc_tf32_k(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of the 16-byte K chunk of (row m, column c) in an operand.
__device__ __forceinline__ int chunk_off(int m, int c)
{
  return (m >> 3) * TC_SBO + c * 128 + (m & 7) * 16;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *m)
{
  asm volatile(
      "{\n\t"
      ".reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t"
      "}\n" ::"r"(tc::smem_addr(m))
      : "memory");
}

__device__ __forceinline__ int ld_vol(const int *p) { return *(const volatile int *)p; }
__device__ __forceinline__ void st_vol(int *p, int v) { *(volatile int *)p = v; }

template <int GEOM>
__global__ void __launch_bounds__(TC_THREADS, 2)
k_fwd3d_band_tc(const Params3D P, const View3D *__restrict__ views, const float *__restrict__ vol,
                long gate_stride, float *__restrict__ sino, long sino_view_stride, int rows, int nuc,
                int ng, int tmem_cols, int a_bytes, int b_bytes, int prof_floats,
                int *__restrict__ err)
{
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ View3D sV;
  __shared__ int s_next, s_claim, s_done, s_freed, s_abort, s_groups;
  __shared__ __align__(8) uint64_t s_full[2], s_mma[2];
  __shared__ uint32_t s_tmem;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nu = P.nu, nv = P.nv;
  const int vi = blockIdx.y;
  const int v0 = blockIdx.x * rows;
  const int v1 = min(v0 + rows, nv);
  unsigned char *A = smraw;                             // ng x a_bytes
  unsigned char *B = A + (size_t)ng * a_bytes;          // ng x b_bytes
  float *profs = reinterpret_cast<float *>(B + (size_t)ng * b_bytes);

  if (threadIdx.x < (int)(sizeof(View3D) / 8))
    reinterpret_cast<double *>(&sV)[threadIdx.x] = reinterpret_cast<const double *>(views + vi)[threadIdx.x];
  if (threadIdx.x == 0) {
    s_next = 0;
    s_claim = 0;
    s_done = 0;
    s_freed = 0;
    s_abort = 0;
    s_groups = 0;
    for (int g = 0; g < 2; ++g) {
      tc::mbar_init(&s_full[g], TC_G);
      tc::mbar_init(&s_mma[g], 1);
    }
    tc::mbar_fence_init();
  }
  {  // operands and profiles start at zero
    float4 *z = reinterpret_cast<float4 *>(smraw);
    const int n4 = (int)(((size_t)ng * (a_bytes + b_bytes) + sizeof(float) * (size_t)TC_PROD * prof_floats) / 16);
    for (int t = threadIdx.x; t < n4; t += TC_THREADS) z[t] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (warp == TC_PROD) tc::tmem_alloc(&s_tmem, (uint32_t)tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = s_tmem;
  const View3D &V = sV;

  if (warp < TC_PROD) {
    // ---------------------------------------------------------------- producers
    float *prof = profs + (size_t)warp * prof_floats;
    const int ncols = P.nx * P.ny;
    const int nchunks = (ncols + 31) >> 5;
    bool quit = false;
    while (!quit) {
      int chunk = 0;
      if (lane == 0) chunk = ld_vol(&s_abort) ? nchunks : atomicAdd(&s_next, 1);
      chunk = __shfl_sync(FULLM, chunk, 0);
      if (chunk >= nchunks) break;
      const int mycol = (chunk << 5) + lane;
      ColGeo<MODEL_CUBIC> c;
      bool hit = false;
      if (mycol < ncols) {
        column_geo<GEOM, MODEL_CUBIC>(P, V, mycol % P.nx, mycol / P.nx, 0, c);
        if (c.bad) atomicOr(err, TRTT_ERR_SOURCE_PLANE);
        hit = !c.bad && c.vax.n > 0 && c.vax.lo + c.vax.n > v0 && c.vax.lo < v1;
      }
      unsigned mask = __ballot_sync(FULLM, hit);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1;
        const ColGeo<MODEL_CUBIC> cc = shfl_colc(c, src);
        const int col = (chunk << 5) + src;
        const int vl = cc.vax.lo, vr = cc.vax.lo + cc.vax.n;
        float wr[2];  // weights of band rows lane and lane + 32 (rows <= 64)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int r = lane + 32 * t, v = v0 + r;
          wr[t] = (r < rows && v >= vl && v < vr && v < v1) ? axis_weight<MODEL_CUBIC>(cc.vax, v - vl, P) : 0.f;
        }
        int lo, hi;
        column_profile<GEOM>(P, V, vol, gate_stride, cc, col, prof, lane, lo, hi);
        __syncwarp();
        if (lo >= hi) continue;  // an all-zero column adds nothing
        // claim a column slot; its buffer must have been consumed ng groups ago
        int s = 0;
        if (lane == 0) s = atomicAdd(&s_claim, 1);
        s = __shfl_sync(FULLM, s, 0);
        const int n = s / TC_G, j = s % TC_G, b = n % ng;
        int stall = 0;
        if (lane == 0 && n >= ng && ld_vol(&s_freed) < n - ng + 1) {
          const uint64_t t0 = tc::global_ns();
          while (ld_vol(&s_freed) < n - ng + 1) {
            if (ld_vol(&s_abort) || tc::global_ns() - t0 > TC_LIMIT_NS) {
              stall = 1;
              break;
            }
          }
        }
        __threadfence_block();
        stall = __shfl_sync(FULLM, stall, 0);
        if (stall) {
          if (lane == 0) {
            atomicOr(err, TRTT_ERR_STALL);
            st_vol(&s_abort, 1);
          }
          quit = true;
          break;
        }
        unsigned char *Ab = A + (size_t)b * a_bytes;
        unsigned char *Bb = B + (size_t)b * b_bytes;
        const int ucells = nuc * 128;
        for (int u = lane; u < ucells; u += 32) {
          float p = 0.f;
          if (u >= lo && u < hi) {
            p = prof[u];
            prof[u] = 0.f;
          }
          const float h = tf32_rna(p), l = tf32_rna(p - h);
          *reinterpret_cast<float4 *>(Ab + chunk_off(u, j)) = make_float4(h, l, h, l);
        }
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int r = lane + 32 * t;
          if (r < rows) {
            const float h = tf32_rna(wr[t]), l = tf32_rna(wr[t] - h);
            *reinterpret_cast<float4 *>(Bb + chunk_off(r, j)) = make_float4(h, h, l, l);
          }
        }
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_full[b]);
      }
    }
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      atomicAdd(&s_done, 1);
    }
  } else {
    // ---------------------------------------------------------------- issuer warp
    const uint32_t idesc = idesc_tf32_k(128, rows);
    const uint32_t a_base = tc::smem_addr(A), b_base = tc::smem_addr(B);
    uint32_t fpar = 0u, mpar = 0u;  // bit b: phase parity of buffer b's barriers
    int n = 0;
    bool stalled = false;
    for (;;) {
      const int b = n % ng;
      // 1: group full; 0: no group n; -1: gave up
      int state = -2;
      bool completed = false;  // the partial last group was completed here
      const uint64_t t0 = tc::global_ns();
      while (state == -2) {
        int st = -2, fill = TC_G;
        if (lane == 0) {
          if (tc::mbar_try_wait(&s_full[b], (fpar >> b) & 1u)) {
            st = 1;
          } else if (ld_vol(&s_abort) || tc::global_ns() - t0 > TC_LIMIT_NS) {
            st = -1;
          } else if (!completed && ld_vol(&s_done) == TC_PROD) {
            // every producer has left its loop, after arriving for each
            // slot it claimed: the claim count is final
            __threadfence_block();
            const int cnt = ld_vol(&s_claim) - TC_G * n;
            if (cnt <= 0) {
              st = 0;
            } else if (cnt < TC_G) {
              st = 2;
              fill = cnt;
            }
          }
        }
        st = __shfl_sync(FULLM, st, 0);
        fill = __shfl_sync(FULLM, fill, 0);
        if (st == 2) {
          // last, partial group: zero the slots nobody filled, then arrive
          // for them so that the group completes
          unsigned char *Ab = A + (size_t)b * a_bytes;
          unsigned char *Bb = B + (size_t)b * b_bytes;
          const int ucells = nuc * 128;
          const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
          for (int j = fill; j < TC_G; ++j) {
            for (int u = lane; u < ucells; u += 32) *reinterpret_cast<float4 *>(Ab + chunk_off(u, j)) = z4;
            for (int r = lane; r < rows; r += 32) *reinterpret_cast<float4 *>(Bb + chunk_off(r, j)) = z4;
          }
          tc::fence_async_smem();
          __syncwarp();
          if (lane == 0)
            for (int j = fill; j < TC_G; ++j) mbar_arrive(&s_full[b]);
          __syncwarp();
          completed = true;
          continue;  // the next try_wait sees the completed phase
        }
        state = st;
      }
      if (state <= 0) {
        stalled = state < 0;
        break;
      }
      tc::fence_after_sync();
      int ok = 1;
      if (lane == 0) {
        const uint32_t ab = a_base + (uint32_t)(b * a_bytes), bb = b_base + (uint32_t)(b * b_bytes);
        for (int uc = 0; uc < nuc; ++uc) {
          const uint32_t d = tbase + (uint32_t)(uc * rows);
#pragma unroll
          for (int t = 0; t < TC_G / 2; ++t) {  // K = 8: columns 2t and 2t + 1
            const uint32_t ko = (uint32_t)(t * 2 * TC_LBO);
            mma_tf32(d, tc::sdesc(ab + (uint32_t)(uc * 16 * TC_SBO) + ko, TC_LBO, TC_SBO),
                     tc::sdesc(bb + ko, TC_LBO, TC_SBO), idesc, (n > 0 || t > 0) ? 1u : 0u);
          }
        }
        tc::mma_commit(&s_mma[b]);
        ok = tc::mbar_wait(&s_mma[b], (mpar >> b) & 1u, TC_LIMIT_NS) ? 1 : 0;
      }
      ok = __shfl_sync(FULLM, ok, 0);
      mpar ^= 1u << b;
      fpar ^= 1u << b;
      ++n;
      if (!ok) {
        stalled = true;
        break;
      }
      if (lane == 0) {
        __threadfence_block();
        st_vol(&s_freed, n);
      }
      __syncwarp();
    }
    if (lane == 0) {
      s_groups = n;
      if (stalled) {
        atomicOr(err, TRTT_ERR_STALL);
        st_vol(&s_abort, 1);
      }
    }
    __syncwarp();
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  // ------------------------------------------------------------------ epilogue
  if (s_groups > 0 && !ld_vol(&s_abort)) {
    float *out = sino + (long)vi * sino_view_stride;
    const int q = warp & 3;
    const int ncb = rows / 16;
    for (int idx = warp >> 2; idx < nuc * ncb; idx += TC_THREADS / 128) {
      const int uc = idx / ncb, cb = idx - uc * ncb;
      float v[16];
      tc::tmem_ld16(tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(uc * rows + cb * 16), v);
      const int u = uc * 128 + 32 * q + lane;
      if (u < nu) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int v_row = v0 + cb * 16 + i;
          if (v_row < v1) out[(long)v_row * nu + u] += v[i];
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == TC_PROD) tc::tmem_dealloc(tbase, (uint32_t)tmem_cols);
}

}  // namespace

int fwd3d_tc_band_rows(int nu, int nv)
{
  (void)nv;
  return tc_shape(nu).rows;
}

}  // namespace trtt

// Host-only query of the kernel's shared-memory plan for an nu-cell-wide
// detector: info = {rows, u chunks, ring groups, TMEM columns, A bytes and B
// bytes of one group, profile floats per warp, dynamic shared memory,
// producer warps, columns per group}; returns -1 (info untouched) if the
// detector is too wide.
extern "C" int trtt_b200_fwd3d_tc_plan_info(int nu, long *info)
{
  const trtt::TcShape t = trtt::tc_shape(nu);
  if (t.rows == 0 || !info) return -1;
  const long v[10] = {t.rows, t.nuc, t.ng, t.tmem_cols, t.a_bytes, t.b_bytes, t.prof_floats,
                      (long)t.smem, trtt::TC_PROD, trtt::TC_G};
  for (int i = 0; i < 10; ++i) info[i] = v[i];
  return 0;
}

namespace trtt {

cudaError_t launch_fwd3d_tc(const Fwd3DLaunch &L, cudaStream_t st)
{
  const TcShape t = tc_shape(L.P.nu);
  if (t.rows == 0) return cudaErrorInvalidValue;
  auto kern = L.P.geom == GEOM_CONE ? k_fwd3d_band_tc<GEOM_CONE> : k_fwd3d_band_tc<GEOM_PARALLEL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
  if (e != cudaSuccess) return e;
  dim3 grid((L.P.nv + t.rows - 1) / t.rows, L.nviews);
  kern<<<grid, TC_THREADS, t.smem, st>>>(L.P, L.views, L.vol, L.gate_stride, L.sino, L.sino_view_stride,
                                         t.rows, t.nuc, t.ng, t.tmem_cols, t.a_bytes, t.b_bytes,
                                         t.prof_floats, L.err);
  return cudaGetLastError();
}

}  // namespace trtt
