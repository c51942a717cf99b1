// Device building blocks of the CS enumeration: the operators' bit arithmetic, the
// fingerprint, warp reductions, mbarrier / bulk-copy / prefetch wrappers and bounded waits.
//
// Operator semantics follow MojtabaValizadeh/ltl-learning-on-gpus, code/ltli6463.cu:
//   ~ :203-204, & :295, | :385, X :468, F :551-556, G :638-645, U :739-771 (both orders).
#pragma once

#include "ltl_kernels.cuh"

namespace ltlg {

constexpr u64 WEYL = 0x9E3779B97F4A7C15ull;
constexpr u64 LENMASK = 0x7FFFFFFFFFFFFFFFull;
constexpr u64 M63 = 0x7FFFFFFFFFFFFFFFull;
constexpr u32 FIELD_PENDING = 0xFFFFFFFFu;
constexpr u32 FIELD_OVERFLOW = 0xFFFFFFFEu;
constexpr unsigned FULL = 0xFFFFFFFFu;

// MurmurHash3's 64-bit finaliser (Appleby, public domain).
__host__ __device__ __forceinline__ u64 fmix64(u64 x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// F: every position at or before the last one where the operand holds, i.e. the
// reference's right smear (ltli6463.cu:553-555) as (2 << msb) - 1.
__device__ __forceinline__ u64 fin_bits(u64 w) { return w ? ((2ull << (63 - __clzll(w))) - 1ull) : 0ull; }

// G: positions after the last position (inside the trace) where the operand fails,
// ltli6463.cu:640-644 (w & ~smear(~w & mask)).  Bit 63 of a mask is never set.
__device__ __forceinline__ u64 glob_bits(u64 w, u64 m) {
    const u64 z = ~w & m;
    return z ? (w & (~0ull << (64 - __clzll(z)))) : w;
}

// x U y.  r_k = y_k | (x_k & r_{k+1}) is a carry chain running from late to early
// positions; bit-reversed it runs upwards, so one 64-bit addition propagates it:
// with A = x|y and B = y (reversed), generate = A&B = y and propagate = A^B = x&~y, and
// the carry into bit j+1 is r at reversed position j.  Positions 0..62 are reversed into
// bits 62..0 (bit 63 of every CS is 0) so the carry into bit 63 holds position 0.  Same
// result as the doubling recurrence of ltli6463.cu:739-752.
__device__ __forceinline__ u64 rev62(u64 v) { return __brevll(v) >> 1; }
__device__ __forceinline__ u64 until_rev(u64 a, u64 yr) {  // a = xr | yr
    return __brevll(((a + yr) ^ a ^ yr) & ~1ull);
}
__device__ __forceinline__ u64 until_bits(u64 x, u64 y) {
    const u64 xr = rev62(x), yr = rev62(y);
    return until_rev(xr | yr, yr);
}

// Unary operator op (OP_NEG, OP_X, OP_F, OP_G) on one word with its length mask m.
__device__ __forceinline__ u64 unary_word(int op, u64 w, u64 m) {
    if (op == OP_NEG) return ~w & m;
    if (op == OP_X) return w >> 1;
    if (op == OP_F) return fin_bits(w);
    return glob_bits(w, m);
}

// Word i (key = (i + 1) * WEYL) of a CS adds to the fingerprint sum:
//   HK 0 (exact keys, verified): (lo(w) + lo(key)) * (hi(w) + hi(key)), one 32x32->64
//        multiply-add in the style of the NH hash (Black et al., UMAC, 1999);
//   HK 1 (64-bit fingerprint, not verified): fmix64(w ^ key), padding words excluded.
template <int HK>
__device__ __forceinline__ u64 hw(u64 w, u64 key, bool valid) {
    if (HK == 0) return (u64)((u32)w + (u32)key) * (u64)((u32)(w >> 32) + (u32)(key >> 32));
    return valid ? fmix64(w ^ key) : 0ull;
}

// Acceptance at position 0 for a pair of words whose traces are positive (p = 1) or not:
// a positive trace where the candidate fails, a negative (or padding) trace where it holds.
__device__ __forceinline__ u32 pmiss2(u64 w0, u64 w1, u64 p0, u64 p1) {
    return (u32)(((~w0 & p0) | (~w1 & p1)) & 1ull);
}
__device__ __forceinline__ u32 nhit2(u64 w0, u64 w1, u64 p0, u64 p1) {
    return (u32)(((w0 & ~p0) | (w1 & ~p1)) & 1ull);
}

__device__ __forceinline__ u64 ld_acquire(const u64 *p) {
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u32 ld_acquire32(const u32 *p) {
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(u64 *p, u64 v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release32(u32 *p, u32 v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ u64 ld_volatile(const u64 *p) { return *(const volatile u64 *)p; }
__device__ __forceinline__ u64 globaltimer() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------- mbarrier + bulk copy
__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(u64 *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(u64 *bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared (no multicast); both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, u32 bytes, u64 *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Bulk prefetch of [src, src + bytes) into L2 (16-byte aligned, size a multiple of 16); no completion.
__device__ __forceinline__ void prefetch_l2(const void *src, u32 bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for phase `parity` of an mbarrier for at most `ns` nanoseconds of globaltimer.
__device__ __forceinline__ bool mbar_wait_for(u64 *bar, u32 parity, u64 ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const u64 t0 = globaltimer();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer() - t0 > ns) return false;
    }
}

// ---------------------------------------------------------------- warp reductions
// Sum v[t] over the warp for NC = 2^K candidates with a reduce-scatter
// (NC - 1 + 5 - K shuffles instead of 5 NC); lane t (< NC) gets candidate t.
template <int NC>
__device__ __forceinline__ u64 reduce_to_lane(u64 (&v)[NC], int lane) {
    constexpr int K = NC == 1 ? 0 : NC == 2 ? 1 : NC == 4 ? 2 : NC == 8 ? 3 : NC == 16 ? 4 : 5;
    static_assert((1 << K) == NC, "NC must be a power of two <= 32");
#pragma unroll
    for (int s = 0; s < K; ++s) {
        const int o = 16 >> s;
        const bool upper = (lane & o) != 0;
        const int half = NC >> (s + 1);
#pragma unroll
        for (int j = 0; j < NC / 2; ++j) {
            if (j < half) {
                const u64 send = upper ? v[j] : v[j + half];
                const u64 keep = upper ? v[j + half] : v[j];
                v[j] = keep + __shfl_xor_sync(FULL, send, o);
            }
        }
    }
    u64 x = v[0];
#pragma unroll
    for (int o = 16 >> K; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    return __shfl_sync(FULL, x, (lane << (5 - K)) & 31);
}

}  // namespace ltlg
