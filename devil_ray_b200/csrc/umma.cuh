// Thin wrappers over the sm_100a tensor-core instructions (tcgen05 /
// UMMA), the tensor memory (TMEM) allocator and shared-memory mbarriers.
//
// Operand layout used throughout (K-major, no swizzle, "interleaved" core
// matrices): an R x K bf16 operand tile is stored as 8-row x 8-element core
// matrices of 128 contiguous bytes; element (r, k) lives at byte
//     (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// with SBO = (K / 8) * 128.  In the UMMA shared-memory descriptor the
// leading-dimension byte offset (LBO) is the distance between the two
// K-adjacent core matrices an instruction reads (128 B) and the
// stride-dimension byte offset (SBO) the distance between 8-row groups.
// One kind::f16 instruction consumes K = 16 (two core matrices along K).
#pragma once

#include <cstdint>
#include "drb_common.cuh"

namespace drb
{
namespace umma
{

DRB_D uint32_t smem_addr (const void *p) { return (uint32_t)__cvta_generic_to_shared (p); }

// byte offset of element (r, k) of a K-major interleaved bf16 tile with K columns
DRB_HD constexpr uint32_t tile_offset (int r, int k, int K)
{
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100 format): start address, LBO and SBO
// in 16-byte units, descriptor version 1, base offset 0, no swizzle.
DRB_D uint64_t desc_kmajor (uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16 with bf16 A and B (both K-major) and
// an fp32 accumulator: c_format F32 (bit 4), a/b format BF16 (bits 7, 10),
// N >> 3 at bit 17, M >> 4 at bit 24.
DRB_HD constexpr uint32_t idesc_bf16_f32 (int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// TMEM allocation (one full warp executes these).
DRB_D void tmem_alloc (uint32_t *smem_result, uint32_t ncols)
{
  asm volatile ("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr (smem_result)),
                "r"(ncols)
                : "memory");
  asm volatile ("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

DRB_D void tmem_dealloc (uint32_t taddr, uint32_t ncols)
{
  asm volatile ("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
DRB_D void mma_bf16 (uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
  asm volatile ("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
                "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
                : "memory");
}

// Arrive on an mbarrier when all previously issued MMAs of this thread finish.
DRB_D void mma_commit (uint64_t *mbar)
{
  asm volatile ("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_addr (mbar))
                : "memory");
}

DRB_D void fence_before_sync () { asm volatile ("tcgen05.fence::before_thread_sync;" ::: "memory"); }
DRB_D void fence_after_sync () { asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Make generic-proxy shared-memory stores visible to the tensor core.
DRB_D void fence_async_smem () { asm volatile ("fence.proxy.async.shared::cta;" ::: "memory"); }

DRB_D void mbar_init (uint64_t *mbar, uint32_t count)
{
  asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr (mbar)), "r"(count) : "memory");
  asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
DRB_D bool mbar_wait (uint64_t *mbar, uint32_t phase, uint32_t max_tries)
{
  const uint32_t a = smem_addr (mbar);
  for (uint32_t i = 0; i < max_tries; ++i)
  {
    uint32_t done;
    asm volatile ("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                  "selp.u32 %0, 1, 0, p;\n\t}\n"
                  : "=r"(done)
                  : "r"(a), "r"(phase)
                  : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive fp32 columns of this thread's TMEM lane.
DRB_D void tmem_ld32 (uint32_t taddr, float (&v)[32])
{
  uint32_t r[32];
  asm volatile ("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                  "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                  "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                  "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                  "=r"(r[30]), "=r"(r[31])
                : "r"(taddr)
                : "memory");
  asm volatile ("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float (r[i]);
}

} // namespace umma
} // namespace drb
