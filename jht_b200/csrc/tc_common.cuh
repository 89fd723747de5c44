// tcgen05 / mbarrier PTX wrappers and the split-BF16 helpers shared by the tensor-core
// kernels (tc_synth.cu, tc_adjoint.cu).  Single-CTA forms only: no cluster multicast.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace tc {

constexpr unsigned kWaitLimit = 1u << 26;  // iteration bound of every mbarrier wait

// ---------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// The same test, but a thread whose phase is not complete is suspended until it completes
// or about hint_ns nanoseconds pass: a waiting warp takes no issue slots from the others.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
constexpr uint32_t kSuspendNs = 20000;  // longest suspension per poll (the watchdog checks between polls)
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: at most kWaitLimit polls and limit_ns of %globaltimer time; returns false
// on timeout (the caller records the error and leaves its loop).  After a first plain test
// the thread sleeps in the barrier between polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;  // the common case: no timer read
    const uint64_t t0 = globaltimer_ns();
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        if (mbar_try_wait_sleep(bar, parity, kSuspendNs)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// A operand from tensor memory (ts form), B from a shared-memory descriptor.
__device__ __forceinline__ void umma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns <-> 8 registers per thread (its own lane's row).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// 32 consecutive columns of this thread's lane, one wait for all of them.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(a), "r"(b), "r"(c),
                 "r"(d)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Shared-memory descriptor, K-major, no swizzle: 8-row x 16-byte core matrices,
// LBO = byte distance between the two 8-element K halves, SBO = between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo) {
    const uint32_t a = smem_u32(p);
    return (uint64_t)((a >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1 (sm100), swizzle none
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with LBO 128, SBO 256
// (K = 16): core matrix (row/8, k/8) at (row/8)*256 + (k/8)*128, row-in-core * 16 + k%8 * 2.
__device__ __forceinline__ uint32_t kmaj_off(int row, int k) {
    return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// x ~ h + m + l with h, m, l BF16: x is rounded to FP32 (the only rounding), then each
// part is the remaining residual rounded to 8 significant bits (to nearest, ties away
// from zero: + 0x8000 on the bit pattern).  Each residual difference is exact in FP32
// (the two operands are within a factor of two), and the last residual has at most 8
// significant bits, so h + m + l == (float)x exactly, with |m| <= 2^-9 |h| and
// |l| <= 2^-17 |h| of either sign: the products the kernels leave out (ml, lm, ll) are
// below 2^-25 of a product and average to zero.  Returns the three parts as FP32 bit
// patterns whose low halves are zero (the BF16 value is the high half).
__device__ __forceinline__ uint32_t bf16_rn_bits(float v) { return (__float_as_uint(v) + 0x8000u) & 0xFFFF0000u; }
__device__ __forceinline__ void split3_bits(double xd, uint32_t &h, uint32_t &m, uint32_t &l) {
    const float x = (float)xd;
    h = bf16_rn_bits(x);
    const float r1 = x - __uint_as_float(h);
    m = bf16_rn_bits(r1);
    const float r2 = r1 - __uint_as_float(m);
    l = __float_as_uint(r2) & 0xFFFF0000u;  // exact: r2 has at most 8 significant bits
}
// The same split as BF16 values (the coefficient and ring-data tiles)
__device__ __forceinline__ void split3(double xd, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l) {
    uint32_t hb, mb, lb;
    split3_bits(xd, hb, mb, lb);
    h = __ushort_as_bfloat16((unsigned short)(hb >> 16));
    m = __ushort_as_bfloat16((unsigned short)(mb >> 16));
    l = __ushort_as_bfloat16((unsigned short)(lb >> 16));
}


__device__ __forceinline__ void rescale(double &u, double &prev, int &sc) {
    if (sc < 0 && fabs(u) > kBig) {
        u *= kScaleDown;
        prev *= kScaleDown;
        sc += 1;
    }
}

// Two FP32 values rounded to BF16 (nearest, ties to even) and packed: lo in the low half.
__device__ __forceinline__ uint32_t cvt_bf16x2(float hi, float lo) {
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// Eight values: the eight FP64 -> FP32 conversions are issued back to back (they run on
// a variable-latency unit, so issuing them together overlaps their latencies), then each
// consecutive pair is split with paired conversions: h = bf16(x), m = bf16(x - h),
// l = x - h - m (exact: at most 8 significant bits remain), packed pk[part][pair] with the
// even value in the low half.
__device__ __forceinline__ void split3_pack8(const double (&v)[8], uint32_t (&pk)[3][4]) {
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = (float)v[i];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float x0 = f[2 * q], x1 = f[2 * q + 1];
        const uint32_t h = cvt_bf16x2(x1, x0);
        const float r10 = x0 - __uint_as_float(h << 16), r11 = x1 - __uint_as_float(h & 0xFFFF0000u);
        const uint32_t m = cvt_bf16x2(r11, r10);
        const float r20 = r10 - __uint_as_float(m << 16), r21 = r11 - __uint_as_float(m & 0xFFFF0000u);
        pk[0][q] = h;
        pk[1][q] = m;
        pk[2][q] = __byte_perm(__float_as_uint(r20), __float_as_uint(r21), 0x7632);
    }
}


// MMA with both operands in shared memory; bulk copy global -> shared (no multicast).
__device__ __forceinline__ void umma_f16_ss(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// One bulk copy (no multicast) into this CTA's shared memory; completes bytes on bar.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Prefetch of a global range into L2 (no shared-memory destination, no completion).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// mbar_wait by every lane of a warp, with one verdict for the warp: a lane that ran out
// makes the whole warp leave together, so no warp-collective instruction after the wait
// can meet a partial warp.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    return __all_sync(0xffffffffu, mbar_wait(bar, parity, limit_ns));
}

}  // namespace tc
}  // namespace jhtb
