// Small inline-PTX helpers for tcgen05 (5th-generation tensor cores), TMEM
// and mbarriers on sm_100a.  Encodings follow the PTX ISA for sm_100a:
//   shared-memory matrix descriptor: start>>4 [0,14), LBO>>4 [16,30),
//     SBO>>4 [32,46), version 1 at [46,48), layout type [61,64) (0 = no swizzle);
//   instruction descriptor (kind::i8 / kind::f16): D format [4,6),
//     A format [7,10), B format [10,13), A/B major [15]/[16], N>>3 [17,23),
//     M>>4 [24,29).
#pragma once

#include <cstdint>

namespace dsplib {
namespace tc {

__device__ __forceinline__ uint32_t smemAddr(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

// K-major operand without swizzle: 8-row core matrices of 16-byte rows.
// lbo = byte distance between the two 16-byte K halves of a core-matrix pair,
// sbo = byte distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t descNoSwizzle(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
   uint64_t d = 0;
   d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
   d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
   d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
   d |= (uint64_t) 1 << 46; // descriptor version for sm_100
   return d;                // layout type 0: no swizzle
}

// K-major operand with 128-byte swizzle: 8-row atoms of 128-byte rows (row
// pitch 128 B), 16-byte chunks permuted by chunk ^= (address bits 7..9);
// sbo = byte distance between consecutive 8-row groups.  The permutation is
// taken from the absolute address, so data stored swizzled by address can be
// read from any 128-byte-aligned start with baseOffset = 0 (measured on B200:
// a non-zero base offset for such starts reads the wrong chunks).
__device__ __forceinline__ uint64_t descSw128(uint32_t saddr, uint32_t sbo, uint32_t baseOffset)
{
   uint64_t d = 0;
   d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
   d |= (uint64_t) 1 << 16; // leading byte offset: unused for swizzled K-major, encoded as 1
   d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
   d |= (uint64_t) 1 << 46;
   d |= (uint64_t) (baseOffset & 7) << 49;
   d |= (uint64_t) 2 << 61; // layout type: 128-byte swizzle
   return d;
}

// Instruction descriptor.  dfmt: 1 = F32, 2 = S32.  afmt/bfmt: kind::i8 -> 0 unsigned, 1 signed;
// kind::f16 -> 0 F16, 1 BF16.  Both operands K-major.
__host__ __device__ constexpr uint32_t idesc(uint32_t dfmt, uint32_t afmt, uint32_t bfmt, uint32_t M, uint32_t N)
{
   return (dfmt << 4) | (afmt << 7) | (bfmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mmaI8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t id, bool accum)
{
   asm volatile("{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
                "l"(adesc), "l"(bdesc), "r"(id), "r"((uint32_t) accum));
}

__device__ __forceinline__ void mmaF16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t id, bool accum)
{
   asm volatile("{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
                "l"(adesc), "l"(bdesc), "r"(id), "r"((uint32_t) accum));
}

// Arrive on an mbarrier once all previously issued tcgen05.mma of this thread complete.
__device__ __forceinline__ void commit(uint64_t *mbar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(mbar))
                : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Make generic-proxy shared-memory writes visible to the tensor core (async proxy).
// Make mbarrier initialisation visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void fenceMbarInit() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbarInit(uint64_t *mbar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint64_t *mbar, uint32_t parity)
{
   uint32_t ok;
   asm volatile("{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, p;\n\t}\n"
                : "=r"(ok)
                : "r"(smemAddr(mbar)), "r"(parity)
                : "memory");
   return ok != 0;
}

// Bounded wait: returns false if the phase did not complete within the limit.
__device__ __forceinline__ bool mbarWait(uint64_t *mbar, uint32_t parity, uint32_t limit = 1u << 22)
{
   for (uint32_t i = 0; i < limit; i++)
      if (mbarTryWait(mbar, parity)) return true;
   return false;
}

// Announce `bytes` of transaction traffic on mbar (this thread's arrival included).
__device__ __forceinline__ void mbarExpectTx(uint64_t *mbar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(mbar)), "r"(bytes)
                : "memory");
}

// Plain arrival of this thread on mbar (release: its earlier shared-memory writes are
// visible to a thread whose wait on mbar completes).
__device__ __forceinline__ void mbarArrive(uint64_t *mbar)
{
   asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(mbar)) : "memory");
}

// Named barrier `id` over the first `n` threads of the CTA (n a multiple of 32), and the
// same with an OR over a predicate of the participating threads.
__device__ __forceinline__ void namedSync(uint32_t id, uint32_t n)
{
   asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ bool namedSyncOr(uint32_t id, uint32_t n, bool v)
{
   uint32_t r;
   asm volatile("{\n\t.reg .pred p, q;\n\t"
                "setp.ne.u32 q, %2, 0;\n\t"
                "bar.red.or.pred p, %1, %3, q;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(r)
                : "r"(id), "r"((uint32_t) v), "r"(n)
                : "memory");
   return r != 0;
}

// Bulk copy (TMA engine, no tensor map) of `bytes` from global memory to this
// CTA's shared memory, completing as transaction bytes on mbar.  Both addresses
// must be 16-byte aligned and bytes a multiple of 16; callers check.
__device__ __forceinline__ void bulkLoad(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smemAddr(dst)),
                "l"(src), "r"(bytes), "r"(smemAddr(mbar))
                : "memory");
}

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned).
__device__ __forceinline__ void cpAsync16(void *dst, const void *src)
{
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smemAddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *slot (shared memory).
__device__ __forceinline__ void tmemAlloc(uint32_t *slot, uint32_t ncols)
{
   asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(slot)),
                "r"(ncols)
                : "memory");
   asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t ncols)
{
   asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns: thread t of the warp receives lane (base lane + t).
__device__ __forceinline__ void tmemLoad8(uint32_t taddr, uint32_t (&r)[8])
{
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(taddr));
}

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp receives lane (base lane + t).
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, uint32_t (&r)[16])
{
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
}

// 32 lanes x 32 consecutive 32-bit columns.
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, uint32_t (&r)[32])
{
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
}

__device__ __forceinline__ void tmemWaitLoad() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

} // namespace tc
} // namespace dsplib
