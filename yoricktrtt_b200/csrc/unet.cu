// unet.cu -- kernels of the learned warm start: a 3-level 3D U-Net whose
// 3x3x3 convolutions (forward, input gradient, weight gradient) run on the
// sm_100a tensor cores (tcgen05.mma, BF16 operands, FP32 accumulators in
// tensor memory), plus its resampling, activation, loss and Adam kernels.
//
// Activation layout, "padded channels-last": a batch of nb volumes of
// d x h x w voxels with C channels (C a multiple of 8) is stored as
//   rows = nb (d+2)(h+2)(w+2) rows of C bf16,
//   row ((v (d+2) + z)(h+2) + y)(w+2) + x, interior z in 1..d, y in 1..h,
//   x in 1..w, and a one-voxel border that is zero and never written.
// With that border the input row of tap (dz, dy, dx) of output row p is
// p + dz (h+2)(w+2) + dy (w+2) + dx for EVERY p, so for a tile of
// consecutive output rows the A operand of each tap is a contiguous run of
// rows of one staged slab: the implicit GEMM needs no im2col copies, only a
// different descriptor start address per tap.  Rows of a tile that fall on
// the border are computed and discarded.
//
// Forward / input-gradient GEMM (k_conv3_fwd), per CTA 128*S output rows:
//   D[row][n] += sum_{tap, k} X[row + off(tap)][k] W[n][tap][k]
//   K loop in stages of (dz, 16 input channels): the stage holds a slab of
//   128*S + 2(w+2) + 2 rows x 16 channels (chunk-major: each 8-channel chunk
//   is a column of 16-byte rows, i.e. a stack of K-major core matrices) and
//   the 9 (dy, dx) weight tiles of that dz; per stage 9*S MMAs of
//   128 x N x 16.  The input gradient is the same kernel run on the output
//   gradient with the weights transposed and flipped (tap -> 26 - tap).
// Weight-gradient GEMM (k_conv3_wgrad), per CTA one (dz, dy) pair and a
// range of rows:
//   dW[co][tap][ci] = sum_row dY[row][co] X[row + off(tap)][ci]
//   with both operands MN-major (the channels-last rows ARE the MN-major
//   core matrices), M = 64 output channels (zero-padded), N = input
//   channels, three accumulators (dx = -1, 0, 1); partial sums per row
//   range are reduced by a second kernel.
//
// Every wait on an mbarrier is bounded in time; a kernel that gives up sets
// a device error word (read by trtt_b200_unet_status), drains its copies,
// frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "runtime.h"
#include "tc100.cuh"
#include "trtt_b200.h"

namespace {

typedef __nv_bfloat16 bf16;

constexpr uint64_t kWaitNs = 2000000000ull;  // bound of every mbarrier wait (2 s)
__device__ int g_unet_err;

struct Grid3 {
  int nb, d, h, w, hp, wp;
  long plane, vol, rows;
};

Grid3 make_grid(int nb, int d, int h, int w)
{
  Grid3 g;
  g.nb = nb; g.d = d; g.h = h; g.w = w;
  g.hp = h + 2; g.wp = w + 2;
  g.plane = (long)g.hp * g.wp;
  g.vol = (long)(d + 2) * g.plane;
  g.rows = (long)nb * g.vol;
  return g;
}

__device__ __forceinline__ bool interior(const Grid3 &g, long p)
{
  if (p < 0 || p >= g.rows) return false;
  const long r = p % g.vol;
  const int z = (int)(r / g.plane);
  const long q = r - (long)z * g.plane;
  const int y = (int)(q / g.wp);
  const int x = (int)(q - (long)y * g.wp);
  return z >= 1 && z <= g.d && y >= 1 && y <= g.h && x >= 1 && x <= g.w;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ float2 unpack_bf16x2(uint32_t u)
{
  __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162 *>(&u);
  return __bfloat1622float2(v);
}

__device__ __forceinline__ float act(float v, float slope) { return v > 0.f ? v : v * slope; }

// ---------------------------------------------------------------------------
// forward / input-gradient convolution
// ---------------------------------------------------------------------------
enum { kFwdAct = 0, kFwdF32 = 1, kFwdHead = 2, kFwdGrad = 3 };

struct FwdArgs {
  const bf16 *x1, *x2;  // input channels [0, c1) from x1, [c1, c1 + c2) from x2
  int c1, c2, groups;   // groups = (c1 + c2) / 16
  const bf16 *wpack;    // [3 groups stages][9 taps][2 chunks][n][8]
  const float *bias;    // [n] or null
  int n, mode;
  float slope;          // activation: v > 0 ? v : slope v (1 = identity)
  void *y, *y2;
  int n1, accumulate;   // kFwdGrad: channels [0, n1) -> y, [n1, n) -> y2
  const float *resid;   // kFwdHead: y[p] = resid[p] + D[p][0] + bias[0]
  Grid3 g;
  long row0;            // first output row of tile 0
  int rh, cs, stage_bytes, nstg;
  uint32_t tmem_cols;
};

// Epilogue of the forward / input-gradient convolution: the S accumulators
// of 128 rows x n columns in tensor memory (warp w reads TMEM lanes
// 32w..32w+31) to bias, activation and the output layout of the mode.
template <int S>
__device__ __forceinline__ void fwd_epilogue(const FwdArgs &a, uint32_t tmem, long m0, int warp, int lane)
{
  const int n = a.n;
#pragma unroll 1
  for (int s = 0; s < S; ++s) {
    const long p = m0 + 128 * s + 32 * warp + lane;
    const bool inside = interior(a.g, p);
#pragma unroll 1
    for (int j = 0; j < n; j += 16) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(s * n + j), v);
      if (!inside) continue;
      if (a.bias && a.mode != kFwdGrad) {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += a.bias[j + i];
      }
      if (a.mode == kFwdAct) {
        uint4 q0, q1;
        q0.x = pack_bf16x2(act(v[0], a.slope), act(v[1], a.slope));
        q0.y = pack_bf16x2(act(v[2], a.slope), act(v[3], a.slope));
        q0.z = pack_bf16x2(act(v[4], a.slope), act(v[5], a.slope));
        q0.w = pack_bf16x2(act(v[6], a.slope), act(v[7], a.slope));
        q1.x = pack_bf16x2(act(v[8], a.slope), act(v[9], a.slope));
        q1.y = pack_bf16x2(act(v[10], a.slope), act(v[11], a.slope));
        q1.z = pack_bf16x2(act(v[12], a.slope), act(v[13], a.slope));
        q1.w = pack_bf16x2(act(v[14], a.slope), act(v[15], a.slope));
        uint4 *dst = reinterpret_cast<uint4 *>(static_cast<bf16 *>(a.y) + p * n + j);
        dst[0] = q0;
        dst[1] = q1;
      } else if (a.mode == kFwdF32) {
        float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(a.y) + p * n + j);
#pragma unroll
        for (int i = 0; i < 4; ++i)
          dst[i] = make_float4(act(v[4 * i], a.slope), act(v[4 * i + 1], a.slope),
                               act(v[4 * i + 2], a.slope), act(v[4 * i + 3], a.slope));
      } else if (a.mode == kFwdHead) {
        if (j == 0) static_cast<float *>(a.y)[p] = a.resid[p] + v[0];
      } else {  // kFwdGrad
        bf16 *base;
        int ld, c0;
        if (j < a.n1) { base = static_cast<bf16 *>(a.y); ld = a.n1; c0 = j; }
        else { base = static_cast<bf16 *>(a.y2); ld = n - a.n1; c0 = j - a.n1; }
        uint4 *dst = reinterpret_cast<uint4 *>(base + p * ld + c0);
        if (a.accumulate) {
          const uint4 o0 = dst[0], o1 = dst[1];
          const uint32_t ow[8] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y, o1.z, o1.w};
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float2 f = unpack_bf16x2(ow[i]);
            v[2 * i] += f.x;
            v[2 * i + 1] += f.y;
          }
        }
        uint4 q0, q1;
        q0.x = pack_bf16x2(v[0], v[1]); q0.y = pack_bf16x2(v[2], v[3]);
        q0.z = pack_bf16x2(v[4], v[5]); q0.w = pack_bf16x2(v[6], v[7]);
        q1.x = pack_bf16x2(v[8], v[9]); q1.y = pack_bf16x2(v[10], v[11]);
        q1.z = pack_bf16x2(v[12], v[13]); q1.w = pack_bf16x2(v[14], v[15]);
        dst[0] = q0;
        dst[1] = q1;
      }
    }
  }
}

template <int S>
__global__ void __launch_bounds__(128) k_conv3_fwd(const FwdArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[4];
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long m0 = a.row0 + (long)blockIdx.x * (128 * S);
  const int T = 3 * a.groups, n = a.n, nstg = a.nstg, pre = nstg - 2;
  const uint32_t sbase = tc::smem_addr(smem);

  if (tid == 0) {
    for (int i = 0; i < nstg; ++i) tc::mbar_init(&mbar[i], 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(&s_taddr, a.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s_taddr;

  auto load = [&](int it, int buf) {
    const int dz = it / a.groups - 1, ch = (it % a.groups) * 16;
    const bf16 *src = a.x1;
    int cst = a.c1, coff = ch;
    if (ch >= a.c1) { src = a.x2; cst = a.c2; coff = ch - a.c1; }
    const long hb = m0 + (long)dz * a.g.plane - a.g.wp - 1;
    const uint32_t hs = sbase + (uint32_t)(buf * a.stage_bytes);
    for (int e = tid; e < 2 * a.rh; e += 128) {
      const int r = e >> 1, c = e & 1;
      const long row = hb + r;
      const bool ok = row >= 0 && row < a.g.rows;
      const bf16 *p = ok ? src + row * cst + coff + c * 8 : src;
      tc::cp16(hs + (uint32_t)(c * a.cs + r * 16), p, ok);
    }
    const uint32_t ws = hs + 2u * a.cs;
    const bf16 *wsrc = a.wpack + (long)it * 9 * n * 16;
    for (int e = tid; e < 9 * n * 2; e += 128) tc::cp16(ws + (uint32_t)e * 16u, wsrc + (long)e * 8, true);
  };

  const uint32_t idesc = tc::idesc_bf16(128, n, 0, 0);
  bool bad = false;
  for (int s = 0; s < pre; ++s) {
    if (s < T) load(s, s);
    tc::cp_commit();
  }
  for (int it = 0; it < T; ++it) {
    const int nxt = it + pre;
    if (nxt < T) {
      if (it >= 2 && !tc::mbar_wait(&mbar[(it - 2) % nstg], ((it - 2) / nstg) & 1, kWaitNs)) bad = true;
      if (!bad) load(nxt, nxt % nstg);
    }
    tc::cp_commit();
    if (pre == 1) tc::cp_wait<1>(); else tc::cp_wait<2>();
    tc::fence_async_smem();
    if (__syncthreads_or(bad)) { bad = true; break; }
    if (tid == 0) {
      tc::fence_after_sync();
      const int buf = it % nstg;
      const uint32_t hs = sbase + (uint32_t)(buf * a.stage_bytes), ws = hs + 2u * a.cs;
      for (int t9 = 0; t9 < 9; ++t9) {
        const int dy = t9 / 3, dx = t9 - 3 * (t9 / 3);
        const uint64_t bd = tc::sdesc(ws + (uint32_t)(t9 * n * 32), (uint32_t)(n * 16), 128u);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const uint64_t ad = tc::sdesc(hs + (uint32_t)((dy * a.g.wp + dx + 128 * s) * 16), (uint32_t)a.cs, 128u);
          tc::mma_bf16(tmem + (uint32_t)(s * n), ad, bd, idesc, (it > 0 || t9 > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(&mbar[buf]);
    }
  }
  if (!bad && T > 0) {
    const int last = T - 1;
    if (!tc::mbar_wait(&mbar[last % nstg], (last / nstg) & 1, kWaitNs)) bad = true;
  }
  bad = __syncthreads_or(bad);

  if (!bad) {
    tc::fence_after_sync();
    fwd_epilogue<S>(a, tmem, m0, warp, lane);
  } else {
    tc::cp_wait_all();
    if (tid == 0) atomicExch(&g_unet_err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, a.tmem_cols);
  }
}

// ---------------------------------------------------------------------------
// forward / input-gradient convolution, TMA staging, warp-specialised
// ---------------------------------------------------------------------------
// Same GEMM, tile and stage layout as k_conv3_fwd, with the slab chunks at a
// 128-byte-aligned stride.  One thread (warp 0) produces: per stage it waits
// until the MMAs of the stage that last used the buffer have read it (the
// buffer's `empty` barrier, signalled by tcgen05.commit), then loads the
// two 8-channel chunks of the slab with 2D tiled TMA copies (boxes of 256
// rows and one box of the remaining rows; rows outside the tensor read as
// zeros) and the 9 weight tiles with one bulk copy, all completing on the
// buffer's `full` barrier as transaction bytes.  One thread (warp 1) waits
// on `full`, issues the stage's 9 S MMAs and commits them to `empty`; after
// the last stage it commits to `acc`, on which every thread waits before
// the epilogue.  The tensor maps cover only this GPU's memory; no copy uses
// cluster multicast.  Every wait is bounded (2 s); a kernel that gives up
// sets the error word, waits for its copies in flight, frees its tensor
// memory and returns.
struct FwdMaps {
  CUtensorMap x1_full, x1_tail, x2_full, x2_tail;  // 8 channels x (256 | tail) rows
  int tail;                                         // rows of the last box (0: none)
};

template <int S>
__global__ void __launch_bounds__(128) k_conv3_fwd_tma(const FwdArgs a, const __grid_constant__ FwdMaps maps)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[4], empty[4], accb;
  __shared__ uint32_t s_taddr;
  __shared__ volatile int s_bad;
  __shared__ int s_issued, s_consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long m0 = a.row0 + (long)blockIdx.x * (128 * S);
  const int T = 3 * a.groups, n = a.n, nstg = a.nstg;
  const uint32_t sbase = tc::smem_addr(smem);

  if (tid == 0) {
    for (int i = 0; i < nstg; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    tc::mbar_init(&accb, 1);
    s_bad = 0;
    s_issued = 0;
    s_consumed = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(&s_taddr, a.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s_taddr;
  const uint32_t stage_tx = (uint32_t)(2 * a.rh * 16 + 288 * n);

  if (tid == 0) {
    // producer
    int it = 0;
    for (; it < T; ++it) {
      const int slot = it % nstg;
      if (it >= nstg && !tc::mbar_wait(&empty[slot], ((it / nstg) - 1) & 1, kWaitNs)) {
        s_bad = 1;
        break;
      }
      if (s_bad) break;
      const int dz = it / a.groups - 1, ch = (it % a.groups) * 16;
      const bool first = ch < a.c1;
      const int coff = first ? ch : ch - a.c1;
      const CUtensorMap *mfull = first ? &maps.x1_full : &maps.x2_full;
      const CUtensorMap *mtail = first ? &maps.x1_tail : &maps.x2_tail;
      const long hb = m0 + (long)dz * a.g.plane - a.g.wp - 1;
      const uint32_t hs = sbase + (uint32_t)(slot * a.stage_bytes);
      tc::mbar_arrive_expect_tx(&full[slot], stage_tx);
      for (int c = 0; c < 2; ++c) {
        for (int r0 = 0; r0 < a.rh; r0 += 256) {
          const bool whole = a.rh - r0 >= 256;
          tc::tma_load_2d(hs + (uint32_t)(c * a.cs + r0 * 16), whole ? mfull : mtail, coff + 8 * c,
                          (int)(hb + r0), &full[slot]);
        }
      }
      tc::bulk_load(hs + 2u * a.cs, a.wpack + (long)it * 9 * n * 16, (uint32_t)(288 * n), &full[slot]);
    }
    s_issued = it;
  } else if (tid == 32) {
    // MMA issuer
    const uint32_t idesc = tc::idesc_bf16(128, n, 0, 0);
    int it = 0;
    for (; it < T; ++it) {
      const int slot = it % nstg;
      if (!tc::mbar_wait(&full[slot], (it / nstg) & 1, kWaitNs)) {
        s_bad = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t hs = sbase + (uint32_t)(slot * a.stage_bytes), ws = hs + 2u * a.cs;
      for (int t9 = 0; t9 < 9; ++t9) {
        const int dy = t9 / 3, dx = t9 - 3 * (t9 / 3);
        const uint64_t bd = tc::sdesc(ws + (uint32_t)(t9 * n * 32), (uint32_t)(n * 16), 128u);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const uint64_t ad = tc::sdesc(hs + (uint32_t)((dy * a.g.wp + dx + 128 * s) * 16), (uint32_t)a.cs, 128u);
          tc::mma_bf16(tmem + (uint32_t)(s * n), ad, bd, idesc, (it > 0 || t9 > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(&empty[slot]);
    }
    tc::mma_commit(&accb);  // arrives once every MMA issued above has completed
    s_consumed = it;
  }
  const bool acc_ok = tc::mbar_wait(&accb, 0, kWaitNs);
  __syncthreads();
  const bool bad = __syncthreads_or(!acc_ok || s_bad);
  if (!bad) {
    tc::fence_after_sync();
    fwd_epilogue<S>(a, tmem, m0, warp, lane);
  } else {
    if (tid == 0) {
      // copies issued for stages the MMAs never consumed
      for (int it = s_consumed; it < s_issued; ++it) tc::mbar_wait(&full[it % nstg], (it / nstg) & 1, kWaitNs);
      atomicExch(&g_unet_err, 1);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, a.tmem_cols);
  }
}

// ---------------------------------------------------------------------------
// forward / input-gradient convolution, TMA staging, persistent
// ---------------------------------------------------------------------------
// Same GEMM, stage layout and TMA copies as k_conv3_fwd_tma, in a persistent
// CTA of 6 warps that walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...:
//   warp 0, one thread: producer.  It streams the stages of all the CTA's
//     tiles through the ring (stage g of the CTA's sequence in buffer
//     g % nstg), waiting on the buffer's `empty` barrier;
//   warp 1, one thread: MMA issuer.  Tile k accumulates in tensor-memory
//     buffer k % 2 (S n columns each); before its first MMA the issuer waits
//     until the epilogue has drained that buffer (`acce`, 4 arrivals), and
//     after its last it commits to `accf`;
//   warps 2-5: epilogue.  Warp w reads TMEM lanes 32 (w % 4) .. +31 of the
//     full buffer, writes the tile's outputs and arrives on `acce`.
// So the copies and MMAs of tile k + 1 overlap the epilogue of tile k.
// Every wait is bounded (2 s); a role that gives up sets the CTA's flag and
// the others stop at their next wait.  Before tensor memory is released,
// every thread waits for a commit issued after the last MMA; copies still
// in flight are waited for, and the error word is set.
template <int S>
__global__ void __launch_bounds__(192) k_conv3_fwd_pers(const FwdArgs a, const __grid_constant__ FwdMaps maps,
                                                       long ntiles)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[4], empty[4], accf[2], acce[2], finb;
  __shared__ uint32_t s_taddr;
  __shared__ volatile int s_bad;
  __shared__ long s_issued, s_consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int T = 3 * a.groups, n = a.n, nstg = a.nstg;
  const uint32_t sbase = tc::smem_addr(smem);
  const uint32_t acc_cols = (uint32_t)(S * n);
  const long nloc = (ntiles - (long)blockIdx.x + gridDim.x - 1) / gridDim.x;  // this CTA's tiles

  if (tid == 0) {
    for (int i = 0; i < nstg; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], 4);
    }
    tc::mbar_init(&finb, 1);
    s_bad = 0;
    s_issued = 0;
    s_consumed = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(&s_taddr, a.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s_taddr;
  const uint32_t stage_tx = (uint32_t)(2 * a.rh * 16 + 288 * n);

  if (tid == 0) {
    // producer
    long g = 0;
    bool ok = true;
    for (long k = 0; k < nloc && ok; ++k) {
      const long m0 = a.row0 + ((long)blockIdx.x + k * gridDim.x) * (128 * S);
      for (int it = 0; it < T; ++it, ++g) {
        const int slot = (int)(g % nstg);
        if (g >= nstg && !tc::mbar_wait(&empty[slot], (uint32_t)((g / nstg) - 1) & 1u, kWaitNs)) {
          s_bad = 1;
          ok = false;
          break;
        }
        if (s_bad) {
          ok = false;
          break;
        }
        const int dz = it / a.groups - 1, ch = (it % a.groups) * 16;
        const bool first = ch < a.c1;
        const int coff = first ? ch : ch - a.c1;
        const CUtensorMap *mfull = first ? &maps.x1_full : &maps.x2_full;
        const CUtensorMap *mtail = first ? &maps.x1_tail : &maps.x2_tail;
        const long hb = m0 + (long)dz * a.g.plane - a.g.wp - 1;
        const uint32_t hs = sbase + (uint32_t)(slot * a.stage_bytes);
        tc::mbar_arrive_expect_tx(&full[slot], stage_tx);
        for (int c = 0; c < 2; ++c) {
          for (int r0 = 0; r0 < a.rh; r0 += 256) {
            const bool whole = a.rh - r0 >= 256;
            tc::tma_load_2d(hs + (uint32_t)(c * a.cs + r0 * 16), whole ? mfull : mtail, coff + 8 * c,
                            (int)(hb + r0), &full[slot]);
          }
        }
        tc::bulk_load(hs + 2u * a.cs, a.wpack + (long)it * 9 * n * 16, (uint32_t)(288 * n), &full[slot]);
      }
    }
    s_issued = g;
  } else if (tid == 32) {
    // MMA issuer
    const uint32_t idesc = tc::idesc_bf16(128, n, 0, 0);
    long g = 0;
    bool ok = true;
    for (long k = 0; k < nloc && ok; ++k) {
      const int b = (int)(k & 1);
      const long u = k >> 1;
      if (u >= 1 && !tc::mbar_wait(&acce[b], (uint32_t)(u - 1) & 1u, kWaitNs)) {
        s_bad = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t acc = tmem + (uint32_t)b * acc_cols;
      for (int it = 0; it < T; ++it, ++g) {
        const int slot = (int)(g % nstg);
        if (s_bad || !tc::mbar_wait(&full[slot], (uint32_t)(g / nstg) & 1u, kWaitNs)) {
          s_bad = 1;
          ok = false;
          break;
        }
        tc::fence_after_sync();
        const uint32_t hs = sbase + (uint32_t)(slot * a.stage_bytes), ws = hs + 2u * a.cs;
        for (int t9 = 0; t9 < 9; ++t9) {
          const int dy = t9 / 3, dx = t9 - 3 * (t9 / 3);
          const uint64_t bd = tc::sdesc(ws + (uint32_t)(t9 * n * 32), (uint32_t)(n * 16), 128u);
#pragma unroll
          for (int s = 0; s < S; ++s) {
            const uint64_t ad = tc::sdesc(hs + (uint32_t)((dy * a.g.wp + dx + 128 * s) * 16), (uint32_t)a.cs, 128u);
            tc::mma_bf16(acc + (uint32_t)(s * n), ad, bd, idesc, (it > 0 || t9 > 0) ? 1u : 0u);
          }
        }
        tc::mma_commit(&empty[slot]);
      }
      if (!ok) break;
      tc::mma_commit(&accf[b]);
    }
    s_consumed = g;
    tc::mma_commit(&finb);  // arrives once every MMA issued above has completed
  } else if (warp >= 2) {
    // epilogue
    const int q = warp & 3;
    for (long k = 0; k < nloc; ++k) {
      const int b = (int)(k & 1);
      const long u = k >> 1;
      const long m0 = a.row0 + ((long)blockIdx.x + k * gridDim.x) * (128 * S);
      // warp-uniform decisions: the tensor-memory loads need the whole warp
      const bool full_ok = tc::mbar_wait(&accf[b], (uint32_t)u & 1u, kWaitNs);
      if (!__all_sync(0xffffffffu, full_ok)) {
        s_bad = 1;
        break;
      }
      tc::fence_after_sync();
      fwd_epilogue<S>(a, tmem + (uint32_t)b * acc_cols, m0, q, lane);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&acce[b]);
      if (__any_sync(0xffffffffu, s_bad != 0)) break;
    }
  }
  const bool fin_ok = tc::mbar_wait(&finb, 0, kWaitNs);
  __syncthreads();
  if (tid == 0 && (s_bad || !fin_ok)) {
    // copies issued for stages the MMAs never consumed
    for (long g = s_consumed; g < s_issued; ++g)
      tc::mbar_wait(&full[g % nstg], (uint32_t)(g / nstg) & 1u, kWaitNs);
    atomicExch(&g_unet_err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, a.tmem_cols);
  }
}

// ---------------------------------------------------------------------------
// weight gradient
// ---------------------------------------------------------------------------

struct WgradArgs {
  const bf16 *dy;       // [rows][cout]
  const bf16 *x1, *x2;  // [rows][c1], [rows][c2]
  int cout, c1, c2, cin;
  float *part;          // [chunks][cout][27][cin]
  Grid3 g;
  long r0, r1;          // rows summed over
  int kt;               // rows (K) per stage: 128 or 256
  int steps;            // kt-row stages per CTA
  int csa, csb, a_bytes, b_bytes, nstg;  // A regions of all stages, then B regions
  uint32_t tmem_cols;
};

__global__ void __launch_bounds__(128) k_conv3_wgrad(const WgradArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[4];
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gidx = blockIdx.x, dzi = gidx / 3, dyi = gidx - 3 * (gidx / 3);
  const long off = (long)(dzi - 1) * a.g.plane + (long)(dyi - 1) * a.g.wp;
  const int KT = a.kt;
  const long qbeg = a.r0 + (long)blockIdx.y * a.steps * KT;
  long rem = a.r1 - qbeg;
  int T = rem <= 0 ? 0 : (int)((rem + KT - 1) / KT);
  if (T > a.steps) T = a.steps;
  const int nstg = a.nstg, pre = nstg - 2, cin = a.cin;
  const int nca = a.cout / 8, ncb = cin / 8;
  const uint32_t sbase = tc::smem_addr(smem);

  if (tid == 0) {
    for (int i = 0; i < nstg; ++i) tc::mbar_init(&mbar[i], 1);
    tc::mbar_fence_init();
  }
  // Only the cout/8 real chunks of the A operand are staged; the M = 64
  // MMAs read the rows above cout from whatever follows them in shared
  // memory (the A regions of all stages come first, then the B regions, and
  // the allocation has a tail where those do not reach 8 chunk strides past
  // the last A region): those accumulator rows are never read back.
  if (warp == 0) tc::tmem_alloc(&s_taddr, a.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s_taddr;

  auto load = [&](int it, int buf) {
    const long q0 = qbeg + (long)it * KT;
    const uint32_t as = sbase + (uint32_t)(buf * a.a_bytes);
    const uint32_t bs = sbase + (uint32_t)(nstg * a.a_bytes + buf * a.b_bytes);
    for (int e = tid; e < KT * nca; e += 128) {
      const int r = e / nca, c = e - nca * (e / nca);
      const long row = q0 + r;
      const bool ok = row < a.r1;
      const bf16 *p = ok ? a.dy + row * a.cout + c * 8 : a.dy;
      tc::cp16(as + (uint32_t)(c * a.csa + r * 16), p, ok);
    }
    const long hb = q0 + off - 1;
    for (int e = tid; e < (KT + 2) * ncb; e += 128) {
      const int r = e / ncb, c = e - ncb * (e / ncb);
      const long row = hb + r;
      const bool ok = row >= 0 && row < a.g.rows;
      const int ch = c * 8;
      const bf16 *p = a.x1;
      if (ok) p = (ch < a.c1) ? a.x1 + row * a.c1 + ch : a.x2 + row * a.c2 + (ch - a.c1);
      tc::cp16(bs + (uint32_t)(c * a.csb + r * 16), p, ok);
    }
  };

  const uint32_t idesc = tc::idesc_bf16(64, cin, 1, 1);
  bool bad = false;
  for (int s = 0; s < pre; ++s) {
    if (s < T) load(s, s);
    tc::cp_commit();
  }
  for (int it = 0; it < T; ++it) {
    const int nxt = it + pre;
    if (nxt < T) {
      if (it >= 2 && !tc::mbar_wait(&mbar[(it - 2) % nstg], ((it - 2) / nstg) & 1, kWaitNs)) bad = true;
      if (!bad) load(nxt, nxt % nstg);
    }
    tc::cp_commit();
    if (pre == 1) tc::cp_wait<1>(); else tc::cp_wait<2>();
    tc::fence_async_smem();
    if (__syncthreads_or(bad)) { bad = true; break; }
    if (tid == 0) {
      tc::fence_after_sync();
      const int buf = it % nstg;
      const uint32_t as = sbase + (uint32_t)(buf * a.a_bytes);
      const uint32_t bs = sbase + (uint32_t)(nstg * a.a_bytes + buf * a.b_bytes);
      // the three accumulators alternate so that consecutive MMAs are independent
#pragma unroll 4
      for (int ks = 0; ks < KT / 16; ++ks) {
        const uint64_t ad = tc::sdesc(as + (uint32_t)(ks * 256), 128u, (uint32_t)a.csa);
        for (int j = 0; j < 3; ++j) {
          const uint64_t bd = tc::sdesc(bs + (uint32_t)((ks * 16 + j) * 16), 128u, (uint32_t)a.csb);
          tc::mma_bf16(tmem + (uint32_t)(j * cin), ad, bd, idesc, (it > 0 || ks > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(&mbar[buf]);
    }
  }
  if (!bad && T > 0) {
    const int last = T - 1;
    if (!tc::mbar_wait(&mbar[last % nstg], (last / nstg) & 1, kWaitNs)) bad = true;
  }
  bad = __syncthreads_or(bad);

  if (!bad) {
    tc::fence_after_sync();
    // M = 64 accumulator: row co = 16 q + r sits in tensor-memory lane 32 q + r
    const int co = 16 * warp + lane;
    const bool mine = lane < 16 && co < a.cout;
    float *dst = a.part + ((long)blockIdx.y * a.cout + (mine ? co : 0)) * 27 * cin;
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      const int tap = gidx * 3 + j;
#pragma unroll 1
      for (int c0 = 0; c0 < cin; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * cin + c0), v);
        if (mine) {
          float4 *o = reinterpret_cast<float4 *>(dst + (long)tap * cin + c0);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (T > 0) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            else o[i] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
      }
    }
  } else {
    tc::cp_wait_all();
    if (tid == 0) atomicExch(&g_unet_err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, a.tmem_cols);
  }
}

// Weight gradient with TMA staging.  The GEMM, the operand layouts (chunk
// columns of 16-byte rows at strides csa / csb, all A regions ahead of the B
// regions) and the MMAs are those of k_conv3_wgrad, in the same order; only
// the staging differs.  Warp specialisation on an mbarrier ring:
//   thread 0: producer.  For each stage it loads the dY rows (A: cout/8
//     chunks of KT rows) and the input rows (B: cin/8 chunks of KT + 2 rows
//     from x1 or x2) as 2D boxes of 8 channels x 128 rows (and a 2-row tail
//     box) of the padded channels-last tensors (tensor maps of this GPU's
//     own buffers, no multicast), completing on the buffer's `full`
//     mbarrier as transaction bytes; it reuses a buffer after its `empty`
//     barrier;
//   thread 32: MMA issuer.  It waits on `full`, issues the stage's MMAs and
//     commits them to `empty`; after the last stage it commits to `finb`;
//   all four warps: the epilogue, after `finb`.
// Rows outside a tensor read as zeros (the halo before its first row).  dY
// rows at or past r1 belong to the last z border plane, zero by the layout,
// or lie past the tensor.  Every wait is bounded (2 s); on a timeout the CTA
// waits (bounded) for the copies it issued, sets the error word, frees its
// tensor memory and leaves its partial sums unwritten.
struct WgradMaps {
  CUtensorMap dy, x1, x2;          // 8 channels x 128 rows
  CUtensorMap x1_tail, x2_tail;    // 8 channels x 2 rows
};

__global__ void __launch_bounds__(128) k_conv3_wgrad_tma(const WgradArgs a, const __grid_constant__ WgradMaps maps)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[4], empty[4], finb;
  __shared__ uint32_t s_taddr;
  __shared__ volatile int s_bad;
  __shared__ int s_issued, s_consumed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gidx = blockIdx.x, dzi = gidx / 3, dyi = gidx - 3 * (gidx / 3);
  const long off = (long)(dzi - 1) * a.g.plane + (long)(dyi - 1) * a.g.wp;
  const int KT = a.kt;
  const long qbeg = a.r0 + (long)blockIdx.y * a.steps * KT;
  const long rem = a.r1 - qbeg;
  int T = rem <= 0 ? 0 : (int)((rem + KT - 1) / KT);
  if (T > a.steps) T = a.steps;
  const int nstg = a.nstg, cin = a.cin;
  const int nca = a.cout / 8, ncb = cin / 8;
  const uint32_t sbase = tc::smem_addr(smem);
  const uint32_t stage_tx = (uint32_t)(16 * (nca * KT + ncb * (KT + 2)));

  if (tid == 0) {
    for (int i = 0; i < nstg; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    tc::mbar_init(&finb, 1);
    s_bad = 0;
    s_issued = 0;
    s_consumed = 0;
    tc::mbar_fence_init();
  }
  // Only the cout/8 real chunks of A are staged; the M = 64 MMAs read the
  // rows above cout from whatever follows them (see k_conv3_wgrad).
  if (warp == 0) tc::tmem_alloc(&s_taddr, a.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = s_taddr;

  if (tid == 0) {
    // producer
    int it = 0;
    for (; it < T; ++it) {
      const int slot = it % nstg;
      if (it >= nstg && !tc::mbar_wait(&empty[slot], (uint32_t)((it / nstg) - 1) & 1u, kWaitNs)) {
        s_bad = 1;
        break;
      }
      if (s_bad) break;
      const long q0 = qbeg + (long)it * KT;
      const long hb = q0 + off - 1;
      const uint32_t as = sbase + (uint32_t)(slot * a.a_bytes);
      const uint32_t bs = sbase + (uint32_t)(nstg * a.a_bytes + slot * a.b_bytes);
      tc::mbar_arrive_expect_tx(&full[slot], stage_tx);
      for (int c = 0; c < nca; ++c)
        for (int r0 = 0; r0 < KT; r0 += 128)
          tc::tma_load_2d(as + (uint32_t)(c * a.csa + r0 * 16), &maps.dy, 8 * c, (int)(q0 + r0), &full[slot]);
      for (int c = 0; c < ncb; ++c) {
        const int ch = 8 * c;
        const bool first = ch < a.c1;
        const CUtensorMap *mb = first ? &maps.x1 : &maps.x2;
        const CUtensorMap *mt = first ? &maps.x1_tail : &maps.x2_tail;
        const int x = first ? ch : ch - a.c1;
        for (int r0 = 0; r0 < KT; r0 += 128)
          tc::tma_load_2d(bs + (uint32_t)(c * a.csb + r0 * 16), mb, x, (int)(hb + r0), &full[slot]);
        tc::tma_load_2d(bs + (uint32_t)(c * a.csb + KT * 16), mt, x, (int)(hb + KT), &full[slot]);
      }
    }
    s_issued = it;
  } else if (tid == 32) {
    // MMA issuer: the MMAs of k_conv3_wgrad, in the same order
    const uint32_t idesc = tc::idesc_bf16(64, cin, 1, 1);
    int it = 0;
    for (; it < T; ++it) {
      const int slot = it % nstg;
      if (s_bad || !tc::mbar_wait(&full[slot], (uint32_t)(it / nstg) & 1u, kWaitNs)) {
        s_bad = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t as = sbase + (uint32_t)(slot * a.a_bytes);
      const uint32_t bs = sbase + (uint32_t)(nstg * a.a_bytes + slot * a.b_bytes);
#pragma unroll 4
      for (int ks = 0; ks < KT / 16; ++ks) {
        const uint64_t ad = tc::sdesc(as + (uint32_t)(ks * 256), 128u, (uint32_t)a.csa);
        for (int j = 0; j < 3; ++j) {
          const uint64_t bd = tc::sdesc(bs + (uint32_t)((ks * 16 + j) * 16), 128u, (uint32_t)a.csb);
          tc::mma_bf16(tmem + (uint32_t)(j * cin), ad, bd, idesc, (it > 0 || ks > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(&empty[slot]);
    }
    s_consumed = it;
    tc::mma_commit(&finb);  // arrives once every MMA issued above has completed
  }
  const bool fin_ok = tc::mbar_wait(&finb, 0, kWaitNs);
  __syncthreads();
  const bool bad = s_bad || !fin_ok;
  if (!bad) {
    tc::fence_after_sync();
    // M = 64 accumulator: row co = 16 q + r sits in tensor-memory lane 32 q + r
    const int co = 16 * warp + lane;
    const bool mine = lane < 16 && co < a.cout;
    float *dst = a.part + ((long)blockIdx.y * a.cout + (mine ? co : 0)) * 27 * cin;
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      const int tap = gidx * 3 + j;
#pragma unroll 1
      for (int c0 = 0; c0 < cin; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * cin + c0), v);
        if (mine) {
          float4 *o = reinterpret_cast<float4 *>(dst + (long)tap * cin + c0);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (T > 0) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            else o[i] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
      }
    }
  } else if (tid == 0) {
    // copies issued for stages the MMAs never consumed
    for (int it = s_consumed; it < s_issued; ++it)
      tc::mbar_wait(&full[it % nstg], (uint32_t)(it / nstg) & 1u, kWaitNs);
    atomicExch(&g_unet_err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, a.tmem_cols);
  }
}

__global__ void k_sum_parts(const float *__restrict__ part, int chunks, long n, float *__restrict__ out)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < chunks; ++c) s += part[(long)c * n + i];
    out[i] = s;
  }
}

// per-channel sum over all rows (bias gradient); rows of the border are zero
__global__ void k_chan_sum(const bf16 *__restrict__ g, long rows, int c, float *__restrict__ out)
{
  extern __shared__ float acc[];
  for (int i = threadIdx.x; i < c; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  const int nch = c / 8;
  float part[8];
  int cur = -1;
  for (int i = 0; i < 8; ++i) part[i] = 0.f;
  // consecutive threads take consecutive 16-byte chunks; each thread keeps
  // the chunk index fixed when the stride is a multiple of nch
  const long total = rows * nch;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int ch = (int)(e % nch);
    if (ch != cur) {
      if (cur >= 0)
        for (int i = 0; i < 8; ++i) atomicAdd(&acc[cur * 8 + i], part[i]), part[i] = 0.f;
      cur = ch;
    }
    const uint4 q = reinterpret_cast<const uint4 *>(g)[e];
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    for (int i = 0; i < 4; ++i) {
      const float2 f = unpack_bf16x2(w[i]);
      part[2 * i] += f.x;
      part[2 * i + 1] += f.y;
    }
  }
  if (cur >= 0)
    for (int i = 0; i < 8; ++i) atomicAdd(&acc[cur * 8 + i], part[i]);
  __syncthreads();
  for (int i = threadIdx.x; i < c; i += blockDim.x) atomicAdd(&out[i], acc[i]);
}

// ---------------------------------------------------------------------------
// weight packing: FP32 master weights w[cout][27][cin] -> BF16 stage tiles
// ---------------------------------------------------------------------------
// forward:   pack[st = dz*G + gi][t9][c][n][k8] = w[n][dz*9 + t9][gi*16 + c*8 + k8],
//            n < npack (rows >= cout zero), G = cin/16
// transpose: the input-gradient weights, n = ci, k = co, tap flipped:
//            pack[st = dz*G + gi][t9][c][n][k8] = w[gi*16 + c*8 + k8][26 - (dz*9 + t9)][n],
//            G = cout_pad/16, n < cin
__global__ void k_pack(const float *__restrict__ w, int cout, int cin, int npack, int kpack, int transpose,
                       bf16 *__restrict__ out)
{
  const int G = kpack / 16;
  const long total = (long)3 * G * 9 * 2 * npack * 8;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int k8 = (int)(e % 8);
    const int nrow = (int)((e / 8) % npack);
    const int c = (int)((e / (8L * npack)) % 2);
    const int t9 = (int)((e / (16L * npack)) % 9);
    const int st = (int)(e / (144L * npack));
    const int dz = st / G, gi = st % G;
    const int tap = dz * 9 + t9, k = gi * 16 + c * 8 + k8;
    float v = 0.f;
    if (!transpose) {
      if (nrow < cout && k < cin) v = w[((long)nrow * 27 + tap) * cin + k];
    } else {
      if (k < cout && nrow < cin) v = w[((long)k * 27 + (26 - tap)) * cin + nrow];
    }
    out[e] = __float2bfloat16_rn(v);
  }
}

// ---------------------------------------------------------------------------
// resampling, activation gradient, input/output conversion, loss, Adam
// ---------------------------------------------------------------------------
__device__ __forceinline__ long prow(const Grid3 &g, int v, int z, int y, int x)
{
  return (((long)v * (g.d + 2) + z) * g.hp + y) * g.wp + x;
}

// thread per (coarse interior voxel, 8-channel chunk).  mode 0: coarse =
// mean of the 8 children; 1: children (+)= coarse / 8 (its adjoint);
// 2: children = coarse (nearest upsampling); 3: coarse (+)= sum of children.
__global__ void k_resample(bf16 *fine, bf16 *coarse, int c, Grid3 gf, Grid3 gc, int mode, int accumulate)
{
  const int nch = c / 8;
  const long total = (long)gc.nb * gc.d * gc.h * gc.w * nch;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % nch);
    long t = e / nch;
    const int x = (int)(t % gc.w); t /= gc.w;
    const int y = (int)(t % gc.h); t /= gc.h;
    const int z = (int)(t % gc.d);
    const int v = (int)(t / gc.d);
    uint4 *cp = reinterpret_cast<uint4 *>(coarse + prow(gc, v, z + 1, y + 1, x + 1) * c) + ch;
    float acc[8];
    if (mode == 0 || mode == 3) {
      for (int i = 0; i < 8; ++i) acc[i] = 0.f;
      for (int k = 0; k < 8; ++k) {
        const long fr = prow(gf, v, 2 * z + 1 + (k >> 2), 2 * y + 1 + ((k >> 1) & 1), 2 * x + 1 + (k & 1));
        const uint4 q = reinterpret_cast<const uint4 *>(fine + fr * c)[ch];
        const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
        for (int i = 0; i < 4; ++i) {
          const float2 f = unpack_bf16x2(w4[i]);
          acc[2 * i] += f.x;
          acc[2 * i + 1] += f.y;
        }
      }
      const float sc = mode == 0 ? 0.125f : 1.f;
      if (accumulate) {
        const uint4 o = *cp;
        const uint32_t w4[4] = {o.x, o.y, o.z, o.w};
        for (int i = 0; i < 4; ++i) {
          const float2 f = unpack_bf16x2(w4[i]);
          acc[2 * i] = acc[2 * i] * sc + f.x;
          acc[2 * i + 1] = acc[2 * i + 1] * sc + f.y;
        }
      } else {
        for (int i = 0; i < 8; ++i) acc[i] *= sc;
      }
      *cp = make_uint4(pack_bf16x2(acc[0], acc[1]), pack_bf16x2(acc[2], acc[3]),
                       pack_bf16x2(acc[4], acc[5]), pack_bf16x2(acc[6], acc[7]));
    } else {
      const uint4 q = *cp;
      const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
      const float sc = mode == 1 ? 0.125f : 1.f;
      for (int i = 0; i < 4; ++i) {
        const float2 f = unpack_bf16x2(w4[i]);
        acc[2 * i] = f.x * sc;
        acc[2 * i + 1] = f.y * sc;
      }
      for (int k = 0; k < 8; ++k) {
        const long fr = prow(gf, v, 2 * z + 1 + (k >> 2), 2 * y + 1 + ((k >> 1) & 1), 2 * x + 1 + (k & 1));
        uint4 *fp = reinterpret_cast<uint4 *>(fine + fr * c) + ch;
        float o[8];
        for (int i = 0; i < 8; ++i) o[i] = acc[i];
        if (accumulate) {
          const uint4 p = *fp;
          const uint32_t w5[4] = {p.x, p.y, p.z, p.w};
          for (int i = 0; i < 4; ++i) {
            const float2 f = unpack_bf16x2(w5[i]);
            o[2 * i] += f.x;
            o[2 * i + 1] += f.y;
          }
        }
        *fp = make_uint4(pack_bf16x2(o[0], o[1]), pack_bf16x2(o[2], o[3]), pack_bf16x2(o[4], o[5]),
                         pack_bf16x2(o[6], o[7]));
      }
    }
  }
}

// g *= (y > 0 ? 1 : slope), 8 channels per thread
__global__ void k_act_grad(bf16 *__restrict__ g, const bf16 *__restrict__ y, long n8, float slope)
{
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n8; e += (long)gridDim.x * blockDim.x) {
    const uint4 q = reinterpret_cast<const uint4 *>(g)[e];
    const uint4 m = reinterpret_cast<const uint4 *>(y)[e];
    const uint32_t gw[4] = {q.x, q.y, q.z, q.w}, mw[4] = {m.x, m.y, m.z, m.w};
    uint32_t o[4];
    for (int i = 0; i < 4; ++i) {
      const float2 a = unpack_bf16x2(gw[i]), b = unpack_bf16x2(mw[i]);
      o[i] = pack_bf16x2(b.x > 0.f ? a.x : a.x * slope, b.y > 0.f ? a.y : a.y * slope);
    }
    reinterpret_cast<uint4 *>(g)[e] = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// dense x[nb][d][h][w] (FP32) -> xb padded [rows][16] BF16 (channel 0 =
// scale x, channels 1..15 zero) and xf padded [rows] FP32 (scale x)
__global__ void k_pad_input(const float *__restrict__ x, bf16 *__restrict__ xb, float *__restrict__ xf, Grid3 g,
                            float scale)
{
  const long total = (long)g.nb * g.d * g.h * g.w;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long t = e;
    const int xx = (int)(t % g.w); t /= g.w;
    const int yy = (int)(t % g.h); t /= g.h;
    const int zz = (int)(t % g.d);
    const int v = (int)(t / g.d);
    const long p = prow(g, v, zz + 1, yy + 1, xx + 1);
    const float val = scale * x[e];
    uint4 *dst = reinterpret_cast<uint4 *>(xb + p * 16);
    dst[0] = make_uint4(pack_bf16x2(val, 0.f), 0u, 0u, 0u);
    dst[1] = make_uint4(0u, 0u, 0u, 0u);
    if (xf) xf[p] = val;
  }
}

// out (padded FP32) -> dense[nb][d][h][w] * scale
__global__ void k_unpad(const float *__restrict__ xf, float *__restrict__ x, Grid3 g, float scale)
{
  const long total = (long)g.nb * g.d * g.h * g.w;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long t = e;
    const int xx = (int)(t % g.w); t /= g.w;
    const int yy = (int)(t % g.h); t /= g.h;
    const int zz = (int)(t % g.d);
    const int v = (int)(t / g.d);
    x[e] = scale * xf[prow(g, v, zz + 1, yy + 1, xx + 1)];
  }
}

// mean squared error against dense target*scale: loss += sum r^2 / count,
// dout[p][0] = 2 r / count (channels 1..15 untouched: zero)
__global__ void k_mse(const float *__restrict__ out, const float *__restrict__ target, bf16 *__restrict__ dout,
                      Grid3 g, float scale, double *__restrict__ loss)
{
  const long total = (long)g.nb * g.d * g.h * g.w;
  const double inv = 1.0 / (double)total;
  double acc = 0.0;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long t = e;
    const int xx = (int)(t % g.w); t /= g.w;
    const int yy = (int)(t % g.h); t /= g.h;
    const int zz = (int)(t % g.d);
    const int v = (int)(t / g.d);
    const long p = prow(g, v, zz + 1, yy + 1, xx + 1);
    const float r = out[p] - scale * target[e];
    acc += (double)r * r;
    if (dout) dout[p * 16] = __float2bfloat16_rn((float)(2.0 * inv) * r);
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) atomicAdd(loss, acc * inv);
  }
}

// dout[p][0] += coef g (dense FP32 g[nb][d][h][w])
__global__ void k_add_out_grad(bf16 *__restrict__ dout, const float *__restrict__ g, Grid3 gr, float coef)
{
  const long total = (long)gr.nb * gr.d * gr.h * gr.w;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    long t = e;
    const int xx = (int)(t % gr.w); t /= gr.w;
    const int yy = (int)(t % gr.h); t /= gr.h;
    const int zz = (int)(t % gr.d);
    const int v = (int)(t / gr.d);
    bf16 *o = dout + prow(gr, v, zz + 1, yy + 1, xx + 1) * 16;
    *o = __float2bfloat16_rn(__bfloat162float(*o) + coef * g[e]);
  }
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long n, float lr, float b1, float b2, float eps, float c1,
                       float c2, float wd)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int grid_for(long n, int threads = 256)
{
  long b = (n + threads - 1) / threads;
  if (b > 148L * 16) b = 148L * 16;
  return (int)(b < 1 ? 1 : b);
}

uint32_t pow2_cols(int n)
{
  uint32_t c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

bool grid_ok(int nb, int d, int h, int w)
{
  return nb > 0 && d > 0 && h > 0 && w > 0 && (long)nb * (d + 2) * (long)(h + 2) * (w + 2) < (1L << 40);
}

constexpr int kSmemPerSM = 228 * 1024;

// pad the dynamic shared memory so that at most 512 / tmem_cols CTAs can
// be resident on one SM (their tensor-memory allocations then always fit)
int residency_smem(int smem, uint32_t tmem_cols)
{
  const int max_ctas = 512 / (int)tmem_cols;
  const int need = kSmemPerSM / (max_ctas + 1) + 1 - 1024;
  return smem < need ? need : smem;
}

// Stage layout of the forward / input-gradient kernel (S = 2 sub-tiles of
// 128 rows per CTA): slab of 128 S + 2 (w+2) + 2 rows per 8-channel chunk,
// two chunks and the 9 tap tiles of the weights per stage.
constexpr int kFwdS = 2;
struct FwdPlan {
  int rh, cs, stage_bytes, nstg, smem;
  long tiles;
  uint32_t tmem_cols;
};

FwdPlan fwd_plan(int n, int groups, const Grid3 &g, int S = kFwdS)
{
  FwdPlan p;
  p.rh = 128 * S + 2 * g.wp + 2;
  p.cs = ((p.rh * 16 + 127) / 128) * 128 + 64;
  p.stage_bytes = ((2 * p.cs + 288 * n + 1023) / 1024) * 1024;
  // a tile with at most 3 stages (16 input channels) has all of them in
  // flight from the start: 3 buffers, and one more CTA per SM
  p.nstg = (3 * groups <= 3 || 4 * p.stage_bytes > 112 * 1024) ? 3 : 4;
  p.tmem_cols = pow2_cols(S * n);
  p.smem = residency_smem(p.nstg * p.stage_bytes, p.tmem_cols);
  const long span = g.rows - 2 * g.plane;
  p.tiles = (span + 128 * S - 1) / (128 * S);
  return p;
}

// Stage layout of the TMA forward kernel: as fwd_plan with the chunk stride
// a multiple of 128 bytes (TMA writes shared memory at 128-byte-aligned
// addresses).
FwdPlan fwd_plan_tma(int n, int groups, const Grid3 &g, int S = kFwdS)
{
  FwdPlan p = fwd_plan(n, groups, g, S);
  p.cs = ((p.rh * 16 + 127) / 128) * 128;
  p.stage_bytes = ((2 * p.cs + 288 * n + 1023) / 1024) * 1024;
  p.nstg = (3 * groups <= 3 || 4 * p.stage_bytes > 112 * 1024) ? 3 : 4;
  p.smem = residency_smem(p.nstg * p.stage_bytes, p.tmem_cols);
  return p;
}

// Stage layout of the persistent TMA forward kernel: tiles of 4 x 128 rows
// where two CTAs still fit on an SM (tensor memory 2 x 4 n columns <= 256,
// and shared memory), else 2 x 128; two tensor-memory accumulators.  *S
// receives the sub-tiles per tile.
FwdPlan fwd_plan_pers(int n, int groups, const Grid3 &g, int *S)
{
  int s = kFwdS;
  if (pow2_cols(2 * 4 * n) <= 256) {
    FwdPlan p4 = fwd_plan_tma(n, groups, g, 4);
    p4.nstg = 4 * p4.stage_bytes <= 112 * 1024 ? 4 : 3;
    if (2 * ((long)residency_smem(p4.nstg * p4.stage_bytes, pow2_cols(2 * 4 * n)) + 2048) <= 227L * 1024) s = 4;
  }
  FwdPlan p = fwd_plan_tma(n, groups, g, s);
  p.tmem_cols = pow2_cols(2 * s * n);
  p.nstg = 4 * p.stage_bytes <= 112 * 1024 ? 4 : 3;
  p.smem = residency_smem(p.nstg * p.stage_bytes, p.tmem_cols);
  *S = s;
  return p;
}

// cuTensorMapEncodeTiled, reached through the runtime (no driver library
// link); null when the driver does not provide it.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled()
{
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of a padded channels-last activation (rows x c BF16): boxes of
// 8 channels x box_rows rows, zeros outside the tensor.
bool act_map(CUtensorMap *m, const void *base, int c, long rows, int box_rows)
{
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)c, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)c * 2};
  const cuuint32_t box[2] = {8u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int g_conv_tma = -1;  // trtt_b200_conv3_set_tma; -1: TMA if the driver can encode tensor maps

// Stage layout of the weight-gradient kernel: 256 rows per stage when two
// CTAs still fit on an SM, else 128; row ranges split into chunks so that
// the grid (9 x chunks) fills about four waves of resident CTAs, each CTA
// running at least 16 stages where the volume is large enough.
struct WgradPlan {
  int kt, csa, csb, a_bytes, b_bytes, nstg, smem;
  long chunks, steps;
  uint32_t tmem_cols;
};

WgradPlan wgrad_plan(int cout, int cin, const Grid3 &g, bool tma = false)
{
  WgradPlan p;
  const int nca = cout / 8, ncb = cin / 8;
  // cp.async: chunk strides padded so that the threads' 16-byte writes of
  // one row spread over the banks; TMA: strides of whole 128-byte lines
  // (its shared-memory destinations are 128-byte aligned)
  const int pad_a = tma ? 0 : nca == 2 ? 64 : nca == 4 ? 32 : 16;
  const int pad_b = tma ? 0 : ncb == 2 ? 64 : ncb == 4 ? 32 : 16;
  p.tmem_cols = pow2_cols(3 * cin);
  for (int kt = 256; kt >= 128; kt /= 2) {
    p.kt = kt;
    p.csa = kt * 16 + pad_a;
    p.csb = (((kt + 2) * 16 + 127) / 128) * 128 + pad_b;
    p.a_bytes = ((nca * p.csa + 127) / 128) * 128;
    p.b_bytes = ((ncb * p.csb + 127) / 128) * 128;
    const int stage = p.a_bytes + p.b_bytes;
    p.nstg = 4 * stage <= 112 * 1024 ? 4 : 3;
    // the last stage's MMAs read 8 chunk strides from its A region
    const int body = p.nstg * stage;
    const int reach = (p.nstg - 1) * p.a_bytes + 8 * p.csa;
    const int total = ((std::max(body, reach) + 1023) / 1024) * 1024;
    p.smem = residency_smem(total, p.tmem_cols);
    if (p.smem <= 112 * 1024) break;
  }
  const long total = (g.rows - 2 * g.plane + p.kt - 1) / p.kt;
  // about four full waves of resident CTAs (shared memory and tensor-memory
  // columns bound the CTAs per SM) over the 9 (dz, dy) groups
  int per_sm = kSmemPerSM / (p.smem + 2048);
  per_sm = std::max(1, std::min(per_sm, 512 / (int)p.tmem_cols));
  long chunks = std::max(1L, 4L * 148 * per_sm / 9);  // 9 chunks never exceed 4 waves
  // at least 16 stages per CTA, unless that leaves fewer than 65 chunks
  chunks = std::min(chunks, std::max(65L, total / 16));
  if (chunks > total) chunks = total;
  if (chunks < 1) chunks = 1;
  p.steps = (total + chunks - 1) / chunks;
  if (p.steps < 1) p.steps = 1;
  p.chunks = (total + p.steps - 1) / p.steps;
  if (p.chunks < 1) p.chunks = 1;
  return p;
}

template <typename K>
cudaError_t set_smem(K kern, int bytes)
{
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace

extern "C" {

int trtt_b200_conv3_forward(const void *x1, int c1, const void *x2, int c2, const void *wpack, int n,
                            const float *bias, int mode, float slope, void *y, void *y2, int n1,
                            int accumulate, const float *resid, int nb, int d, int h, int w, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!x1 || !wpack || !y) return fail("conv3_forward: null pointer");
  if (c1 <= 0 || c1 % 16 || c2 < 0 || c2 % 16 || (c2 > 0 && !x2))
    return fail("conv3_forward: input channels must be multiples of 16");
  if (n < 16 || n > 256 || n % 16) return fail("conv3_forward: output channels must be a multiple of 16 in [16, 256]");
  if (mode < kFwdAct || mode > kFwdGrad) return fail("conv3_forward: bad mode");
  if (mode == kFwdHead && !resid) return fail("conv3_forward: head mode needs the residual input");
  if (mode == kFwdGrad && (n1 < 0 || n1 > n || n1 % 16 || (n1 < n && !y2)))
    return fail("conv3_forward: bad channel split");
  if (!grid_ok(nb, d, h, w)) return fail("conv3_forward: bad grid");
  constexpr int S = kFwdS;
  FwdArgs a;
  a.x1 = static_cast<const bf16 *>(x1);
  a.x2 = static_cast<const bf16 *>(x2);
  a.c1 = c1; a.c2 = c2; a.groups = (c1 + c2) / 16;
  a.wpack = static_cast<const bf16 *>(wpack);
  a.bias = bias; a.n = n; a.mode = mode; a.slope = slope;
  a.y = y; a.y2 = y2; a.n1 = mode == kFwdGrad ? n1 : n; a.accumulate = accumulate;
  a.resid = resid;
  a.g = make_grid(nb, d, h, w);
  a.row0 = a.g.plane;
  // staging: 0 cp.async, 1 TMA per tile, 2 TMA persistent (two tensor-memory
  // accumulators: 2 S n columns must fit in 512); automatic: the persistent
  // kernel where it applies, else TMA per tile, else cp.async (forward pass
  // of the 128^3 U-Net: 1.03 / 1.37 / 1.73 ms)
  int tma = g_conv_tma < 0 ? (encode_tiled() ? 2 : 0) : g_conv_tma;
  if (tma == 2 && pow2_cols(2 * S * n) > 512) tma = 1;
  if (a.g.rows < 256) tma = 0;  // tensors shorter than one 256-row box: cp.async
  // persistent kernel: tiles of 4 x 128 rows where two CTAs still fit on an
  // SM (fwd_plan_pers).  The slab of a tile overlaps the next tile's by
  // 2 (w+2) + 2 rows, so longer tiles stage each input row fewer times (1.5
  // instead of 2 slab rows per output row at 128^3) and fetch each stage's
  // weights for twice the rows (forward pass 1.18 -> 1.03 ms)
  int sp = S;
  if (tma) {
    const FwdPlan pl = tma == 2 ? fwd_plan_pers(n, a.groups, a.g, &sp) : fwd_plan_tma(n, a.groups, a.g);
    const bool s4 = sp == 4;
    a.rh = pl.rh;
    a.cs = pl.cs;
    a.stage_bytes = pl.stage_bytes;
    a.nstg = pl.nstg;
    a.tmem_cols = pl.tmem_cols;
    if (pl.smem > 227 * 1024) return fail("conv3_forward: volume rows too long for the staged slab");
    if (pl.tiles <= 0 || pl.tiles > 0x7FFFFFFFL) return fail("conv3_forward: bad tile count");
    if ((reinterpret_cast<uintptr_t>(x1) & 15) || (c2 && (reinterpret_cast<uintptr_t>(x2) & 15)) ||
        (reinterpret_cast<uintptr_t>(wpack) & 15))
      return fail("conv3_forward: TMA staging needs 16-byte aligned tensors");
    FwdMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    maps.tail = pl.rh % 256;
    const int tail = maps.tail ? maps.tail : 256;
    bool ok = act_map(&maps.x1_full, x1, c1, a.g.rows, 256) && act_map(&maps.x1_tail, x1, c1, a.g.rows, tail);
    if (c2) ok = ok && act_map(&maps.x2_full, x2, c2, a.g.rows, 256) && act_map(&maps.x2_tail, x2, c2, a.g.rows, tail);
    if (!ok) return fail("conv3_forward: tensor map encoding failed");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (tma == 2) {
      auto kern = s4 ? k_conv3_fwd_pers<4> : k_conv3_fwd_pers<S>;
      TRTT_CK(set_smem(kern, pl.smem));
      // all of the SM's unified memory as shared memory, so that the
      // occupancy below (and the launch) can hold several CTAs
      TRTT_CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      int dev = 0, sms = 0, occ = 0;
      TRTT_CK(cudaGetDevice(&dev));
      TRTT_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      TRTT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 192, pl.smem));
      // the query answered 1 where two CTAs fit (measured: 1.96 ms per
      // forward pass of the 128^3 U-Net at one CTA per SM, 1.18 ms at two);
      // CTAs per SM by shared memory (plus the static and reserved bytes)
      // and tensor memory, which residency_smem keeps consistent
      const int by_smem = (int)((227L * 1024) / ((long)pl.smem + 2048));
      occ = std::max(occ, std::min(by_smem, (int)(512u / pl.tmem_cols)));
      if (occ < 1) return fail("conv3_forward: the persistent kernel does not fit on an SM");
      const long grid = std::min<long>(pl.tiles, (long)sms * occ);
      kern<<<(unsigned)grid, 192, pl.smem, st>>>(a, maps, pl.tiles);
    } else {
      TRTT_CK(set_smem(k_conv3_fwd_tma<S>, pl.smem));
      k_conv3_fwd_tma<S><<<(unsigned)pl.tiles, 128, pl.smem, st>>>(a, maps);
    }
    count_launch();
    TRTT_CK(cudaGetLastError());
    return 0;
  }
  const FwdPlan pl = fwd_plan(n, a.groups, a.g);
  a.rh = pl.rh;
  a.cs = pl.cs;
  a.stage_bytes = pl.stage_bytes;
  a.nstg = pl.nstg;
  a.tmem_cols = pl.tmem_cols;
  const int smem = pl.smem;
  if (smem > 227 * 1024) return fail("conv3_forward: volume rows too long for the staged slab");
  const long tiles = pl.tiles;
  if (tiles <= 0 || tiles > 0x7FFFFFFFL) return fail("conv3_forward: bad tile count");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  TRTT_CK(set_smem(k_conv3_fwd<S>, smem));
  k_conv3_fwd<S><<<(unsigned)tiles, 128, smem, st>>>(a);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_conv3_set_tma(int on)
{
  using namespace trtt;
  clear_error();
  if (on > 0 && !encode_tiled()) return fail("conv3_set_tma: the driver provides no tensor-map encoder");
  if (on > 2) return fail("conv3_set_tma: mode must be -1 (automatic), 0, 1 or 2");
  g_conv_tma = on < 0 ? -1 : on;
  return 0;
}

int trtt_b200_conv3_plan_info(int which, int cin, int cout, int nb, int d, int h, int w, long *info)
{
  using namespace trtt;
  clear_error();
  if (!info || !grid_ok(nb, d, h, w) || cin <= 0 || cout <= 0 || cin % 16 || cout % 16)
    return fail("conv3_plan_info: bad arguments");
  const Grid3 g = make_grid(nb, d, h, w);
  if (which == 0) {
    const FwdPlan p = fwd_plan(cout, cin / 16, g);
    const long v[] = {kFwdS, p.rh, p.cs, p.stage_bytes, p.nstg, p.smem, p.tmem_cols, p.tiles};
    for (int i = 0; i < 8; ++i) info[i] = v[i];
    return 0;
  }
  if (which == 1 || which == 3) {
    const WgradPlan p = wgrad_plan(cout, cin, g, which == 3);
    const long v[] = {p.kt, p.csa, p.csb, p.a_bytes, p.b_bytes, p.nstg, p.smem, p.tmem_cols, p.chunks, p.steps};
    for (int i = 0; i < 10; ++i) info[i] = v[i];
    return 0;
  }
  if (which == 2) {
    int S = kFwdS;
    const FwdPlan p = fwd_plan_pers(cout, cin / 16, g, &S);
    const long v[] = {S, p.rh, p.cs, p.stage_bytes, p.nstg, p.smem, p.tmem_cols, p.tiles};
    for (int i = 0; i < 8; ++i) info[i] = v[i];
    return 0;
  }
  return fail("conv3_plan_info: which must be 0 (forward, cp.async), 1 (weight gradient, cp.async), "
              "2 (forward, persistent TMA) or 3 (weight gradient, TMA)");
}

size_t trtt_b200_conv3_wgrad_scratch(int cout, int cin, int nb, int d, int h, int w)
{
  if (!grid_ok(nb, d, h, w) || cout <= 0 || cin <= 0 || cout % 8 || cin % 8) return 0;
  // enough for either staging
  const Grid3 g = make_grid(nb, d, h, w);
  const long chunks = std::max(wgrad_plan(cout, cin, g, false).chunks, wgrad_plan(cout, cin, g, true).chunks);
  return (size_t)chunks * cout * 27 * cin * sizeof(float);
}

int trtt_b200_conv3_wgrad(const void *dy, int cout, const void *x1, int c1, const void *x2, int c2, float *dw,
                          float *db, void *scratch, size_t scratch_bytes, int nb, int d, int h, int w,
                          void *stream)
{
  using namespace trtt;
  clear_error();
  if (!dy || !x1 || !dw || !scratch) return fail("conv3_wgrad: null pointer");
  const int cin = c1 + c2;
  if (cout <= 0 || cout > 64 || cout % 16) return fail("conv3_wgrad: output channels must be 16, 32, 48 or 64");
  if (c1 <= 0 || c1 % 16 || c2 < 0 || c2 % 16 || (c2 > 0 && !x2) || 3 * cin > 512)
    return fail("conv3_wgrad: input channels must be multiples of 16 with 3 cin <= 512");
  if (!grid_ok(nb, d, h, w)) return fail("conv3_wgrad: bad grid");
  WgradArgs a;
  a.dy = static_cast<const bf16 *>(dy);
  a.x1 = static_cast<const bf16 *>(x1);
  a.x2 = static_cast<const bf16 *>(x2);
  a.cout = cout; a.c1 = c1; a.c2 = c2; a.cin = cin;
  a.g = make_grid(nb, d, h, w);
  a.r0 = a.g.plane;
  a.r1 = a.g.rows - a.g.plane;
  // staging: TMA unless cp.async is asked for (trtt_b200_conv3_set_tma(0)) or
  // the driver has no tensor-map encoder; rows must be addressable by the
  // 32-bit coordinates of a tensor copy, the tensors 16-byte aligned
  const bool tma = g_conv_tma != 0 && encode_tiled() && a.g.rows >= 256 && a.g.rows + 512 < 0x7FFFFFFFL &&
                   !(reinterpret_cast<uintptr_t>(dy) & 15) && !(reinterpret_cast<uintptr_t>(x1) & 15) &&
                   !(c2 && (reinterpret_cast<uintptr_t>(x2) & 15));
  const WgradPlan pl = wgrad_plan(cout, cin, a.g, tma);
  if (pl.steps > 0x7FFFFFFFL) return fail("conv3_wgrad: too many rows");
  const long chunks = pl.chunks;
  a.kt = pl.kt;
  a.steps = (int)pl.steps;
  const size_t need = (size_t)chunks * cout * 27 * cin * sizeof(float);
  if (scratch_bytes < need) return fail("conv3_wgrad: scratch too small");
  a.part = static_cast<float *>(scratch);
  a.csa = pl.csa;
  a.csb = pl.csb;
  a.a_bytes = pl.a_bytes;
  a.b_bytes = pl.b_bytes;
  a.nstg = pl.nstg;
  a.tmem_cols = pl.tmem_cols;
  const int smem = pl.smem;
  if (smem > 227 * 1024) return fail("conv3_wgrad: stage too large");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 grid(9, (unsigned)chunks);
  if (tma) {
    WgradMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    bool ok = act_map(&maps.dy, dy, cout, a.g.rows, 128) && act_map(&maps.x1, x1, c1, a.g.rows, 128) &&
              act_map(&maps.x1_tail, x1, c1, a.g.rows, 2);
    if (c2) ok = ok && act_map(&maps.x2, x2, c2, a.g.rows, 128) && act_map(&maps.x2_tail, x2, c2, a.g.rows, 2);
    if (!ok) return fail("conv3_wgrad: tensor map encoding failed");
    TRTT_CK(set_smem(k_conv3_wgrad_tma, smem));
    k_conv3_wgrad_tma<<<grid, 128, smem, st>>>(a, maps);
  } else {
    TRTT_CK(set_smem(k_conv3_wgrad, smem));
    k_conv3_wgrad<<<grid, 128, smem, st>>>(a);
  }
  const long nw = (long)cout * 27 * cin;
  k_sum_parts<<<grid_for(nw), 256, 0, st>>>(a.part, (int)chunks, nw, dw);
  count_launch(2);
  if (db) {
    TRTT_CK(cudaMemsetAsync(db, 0, sizeof(float) * cout, st));
    k_chan_sum<<<148 * 4, 256, sizeof(float) * cout, st>>>(a.dy, a.g.rows, cout, db);
    count_launch();
  }
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_conv3_pack(const float *w, int cout, int cin, int transpose, void *wpack, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!w || !wpack) return fail("conv3_pack: null pointer");
  if (cout <= 0 || cin <= 0 || cin % 16) return fail("conv3_pack: cin must be a multiple of 16");
  const int coutp = (cout + 15) / 16 * 16;
  const int npack = transpose ? cin : coutp;
  const int kpack = transpose ? coutp : cin;
  const long total = (long)27 * npack * kpack;
  k_pack<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, cout, cin, npack, kpack, transpose,
                                                                         static_cast<bf16 *>(wpack));
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_resample(void *fine, void *coarse, int c, int nb, int d, int h, int w, int mode,
                            int accumulate, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!fine || !coarse) return fail("unet_resample: null pointer");
  if (c <= 0 || c % 8 || d % 2 || h % 2 || w % 2 || mode < 0 || mode > 3)
    return fail("unet_resample: channels must be a multiple of 8 and the fine grid even");
  if (!grid_ok(nb, d, h, w)) return fail("unet_resample: bad grid");
  const Grid3 gf = make_grid(nb, d, h, w), gc = make_grid(nb, d / 2, h / 2, w / 2);
  const long total = (long)nb * (d / 2) * (h / 2) * (w / 2) * (c / 8);
  k_resample<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<bf16 *>(fine), static_cast<bf16 *>(coarse), c, gf, gc, mode, accumulate);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_act_grad(void *g, const void *y, long rows, int c, float slope, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!g || !y || rows <= 0 || c <= 0 || c % 8) return fail("unet_act_grad: bad arguments");
  const long n8 = rows * (c / 8);
  k_act_grad<<<grid_for(n8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<bf16 *>(g), static_cast<const bf16 *>(y), n8, slope);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_pad_input(const float *x, void *xb, float *xf, float scale, int nb, int d, int h, int w,
                             void *stream)
{
  using namespace trtt;
  clear_error();
  if (!x || !xb || !grid_ok(nb, d, h, w)) return fail("unet_pad_input: bad arguments");
  const Grid3 g = make_grid(nb, d, h, w);
  k_pad_input<<<grid_for((long)nb * d * h * w), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      x, static_cast<bf16 *>(xb), xf, g, scale);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_unpad(const float *xf, float *x, float scale, int nb, int d, int h, int w, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!x || !xf || !grid_ok(nb, d, h, w)) return fail("unet_unpad: bad arguments");
  const Grid3 g = make_grid(nb, d, h, w);
  k_unpad<<<grid_for((long)nb * d * h * w), 256, 0, static_cast<cudaStream_t>(stream)>>>(xf, x, g, scale);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_mse(const float *out, const float *target, void *dout, float scale, double *loss, int nb,
                       int d, int h, int w, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!out || !target || !loss || !grid_ok(nb, d, h, w)) return fail("unet_mse: bad arguments");
  const Grid3 g = make_grid(nb, d, h, w);
  k_mse<<<grid_for((long)nb * d * h * w), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      out, target, static_cast<bf16 *>(dout), g, scale, loss);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_add_output_grad(void *dout, const float *g, float coef, int nb, int d, int h, int w,
                                   void *stream)
{
  using namespace trtt;
  clear_error();
  if (!dout || !g || !grid_ok(nb, d, h, w)) return fail("unet_add_output_grad: bad arguments");
  const Grid3 gr = make_grid(nb, d, h, w);
  k_add_out_grad<<<grid_for((long)nb * d * h * w), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<bf16 *>(dout), g, gr, coef);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_adam(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
                   int step, float weight_decay, void *stream)
{
  using namespace trtt;
  clear_error();
  if (!w || !g || !m || !v || n <= 0 || step < 1) return fail("adam: bad arguments");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2,
                                                                     weight_decay);
  count_launch();
  TRTT_CK(cudaGetLastError());
  return 0;
}

int trtt_b200_unet_status(void *stream)
{
  using namespace trtt;
  clear_error();
  int e = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  TRTT_CK(cudaMemcpyFromSymbolAsync(&e, g_unet_err, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
  TRTT_CK(cudaStreamSynchronize(st));
  if (e) {
    const int zero = 0;
    TRTT_CK(cudaMemcpyToSymbolAsync(g_unet_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st));
    TRTT_CK(cudaStreamSynchronize(st));
    return fail("tensor-core convolution gave up waiting for its MMAs (time limit reached)");
  }
  return 0;
}

}  // extern "C"
