// tc100.cuh -- sm_100a building blocks written as inline PTX for the
// tensor-core convolutions: shared-memory matrix descriptors and instruction
// descriptors of tcgen05.mma (kind::f16 with BF16 operands and FP32
// accumulators in tensor memory), tensor-memory allocation and loads,
// mbarriers with time-bounded waits, and 16-byte cp.async copies.
//
// Operand layouts are the "no swizzle" canonical layouts: a core matrix is
// 8 rows x 16 bytes stored as 128 contiguous bytes.
//   K-major  (row = M or N index, 16 bytes = 8 consecutive K elements):
//     element (r, k) at start + (r/8)*SBO + (r%8)*16 + (k/8)*LBO + (k%8)*2
//   MN-major (16 bytes = 8 consecutive M/N elements, row = K index):
//     element (r, k) at start + (r/8)*SBO + (r%8)*2  + (k/8)*LBO + (k%8)*16
#pragma once

#include <cstdint>

namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle):
//   bits  0-13 start address >> 4      bits 16-29 leading byte offset >> 4
//   bits 32-45 stride byte offset >> 4 bits 46-47 version (1)
//   bits 49-51 base offset (0)         bits 61-63 layout (0 = no swizzle)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16 with BF16 A and B and FP32 D:
//   bits 4-5 D format (1 = F32), 7-9 A format (1 = BF16), 10-12 B format,
//   bit 15 A major (0 = K, 1 = MN), bit 16 B major, 17-22 N >> 3, 24-28 M >> 4.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
  const uint32_t z = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z),
        "r"(z)
      : "memory");
}

// Arrive on `mbar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Make this thread's generic-proxy shared-memory writes visible to the
// tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tensor memory: allocation by one whole warp; the base address is written
// to shared memory.  ncols is a power of two >= 32.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread i of the warp receives
// lane (taddr.lane + i), columns taddr.col .. taddr.col + 15.  The wait is
// tied to the registers so that no use is scheduled before it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                 "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                 "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// mbarriers --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase of parity `parity`; gives up (returns false) after
// `limit_ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t parity, uint64_t limit_ns)
{
  if (mbar_try_wait(m, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(m, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// Tensor memory accelerator (TMA) -----------------------------------------
// All copies here read this GPU's own global memory into this CTA's shared
// memory (no cluster multicast).  Completion is signalled on an mbarrier as
// transaction bytes.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *m, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)), "r"(bytes)
               : "memory");
}
// Plain arrive (count 1) on an mbarrier of this CTA.
__device__ __forceinline__ void mbar_arrive(uint64_t *m)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(m)) : "memory");
}
// 2D tiled load of the tensor map's box at element coordinates (x, y), x
// the innermost dimension (x * element size a multiple of 16 bytes).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void *tmap, int x, int y, uint64_t *mbar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_addr(mbar))
      : "memory");
}
// Contiguous copy of `bytes` (a multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_addr(mbar))
               : "memory");
}

// cp.async ---------------------------------------------------------------
// 16-byte global -> shared copy; `valid` false writes 16 zero bytes (the
// source is not read).
__device__ __forceinline__ void cp16(uint32_t dst, const void *src, bool valid)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

}  // namespace tc
