// sht_tc.cuh -- thin inline-PTX wrappers for the sm_100a tensor-core path:
// tcgen05 TMEM allocation, MMA issue and commit, TMEM loads, mbarriers with
// bounded waits, and the UMMA shared-memory / instruction descriptors.
//
// Descriptor encodings (tcgen05 "shared memory descriptor" and "instruction
// descriptor" of the PTX ISA):
//   smem desc: [0,14) start >> 4, [16,30) leading-dim byte offset >> 4,
//              [32,46) stride-dim byte offset >> 4, [46,48) version = 1,
//              [49,52) base offset, [52] lbo mode, [61,64) swizzle (0 = none)
//   instr desc (kind::f16): [4,6) D format (1 = F32), [7,10) A format
//              (1 = BF16), [10,13) B format, [15] A major, [16] B major
//              (0 = K-major), [17,23) N >> 3, [24,29) M >> 4.
// K-major operands without swizzle use the interleaved canonical layout:
// core matrices of 8 rows x 16 bytes (rows 16 B apart).  Here the two core
// matrices along K of one MMA are LBO apart, and consecutive groups of 8 rows
// are SBO apart.
#pragma once

#include <cstdint>

namespace sht {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // version
  return d;                 // base offset 0, lbo mode 0, no swizzle
}

// BF16 x BF16 -> F32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// signed 8-bit x signed 8-bit -> S32 (kind::i8), both operands K-major:
// D format 2 (S32) at [4,6), A and B format 1 (signed 8-bit) at [7,10) and
// [10,13), no saturation.
__host__ __device__ constexpr uint32_t idesc_s8_s32(int M, int N)
{
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------------- TMEM
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(dst_smem)), "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::); }
// make generic-proxy shared-memory writes visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::); }
// generic-proxy global stores of this thread made visible to later bulk copies
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// D[tmem] (+)= A[smem] * B[smem]^T with 8-bit integer operands and exact
// 32-bit integer accumulation, issued by one thread
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// arrive on an mbarrier once all previously issued tcgen05 ops of this thread complete
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(mbar)));
}

// 32 lanes x 32 bits, 16 consecutive columns -> 16 registers per thread
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// 32 lanes x 32 bits, 8 consecutive columns -> 8 registers per thread
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8])
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
// 32 lanes x 32 bits, 4 consecutive columns -> 4 registers per thread
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4])
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::); }

// ------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mbar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::); }

// One thread announces `bytes` of asynchronous copies on the barrier and
// arrives (release: shared-memory stores made before it are visible to the
// threads that wait on the phase).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(mbar)), "r"(bytes) : "memory");
}

// Plain arrive (release at CTA scope: this thread's shared-memory stores made
// before it are visible to the threads that wait on the phase).
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(mbar)) : "memory");
}

// One poll of the phase with parity `parity` (acquire when it returns true).
__device__ __forceinline__ bool mbar_try(uint32_t mbar_addr, uint32_t parity)
{
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar_addr), "r"(parity)
      : "memory");
  return done != 0;
}

// The same with a suspend-time hint: the thread may sleep up to `hint_ns`
// inside the call until the phase completes, instead of spinning.
__device__ __forceinline__ bool mbar_try_sleep(uint32_t mbar_addr, uint32_t parity, uint32_t hint_ns)
{
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar_addr), "r"(parity), "r"(hint_ns)
      : "memory");
  return done != 0;
}

// Bulk copy global -> shared of `bytes` (a multiple of 16; both addresses
// 16-byte aligned), completing on the barrier (plain copy, no multicast).
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src, uint32_t bytes, uint64_t *mbar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst_smem)),
               "l"(src), "r"(bytes), "r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase with parity `parity` to complete.  Gives up once
// `limit_ns` of wall time has passed (try_wait itself may suspend for a
// system-defined time per poll, so the bound is on time, not on polls) and
// returns false; the caller records the timeout and unwinds.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint64_t limit_ns)
{
  const uint32_t a = smem_addr(mbar);
  const uint64_t t0 = globaltimer_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity));
    if (done) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

}  // namespace tc
}  // namespace sht
