// Characteristic-set (CS) enumeration kernels for sm_100a.
//
// One persistent launch per cost level drains a device work queue of items cut
// from the level's (operator, split) blocks.  A binary item stages a tile of
// left-operand CSs in shared memory with one bulk copy (cp.async.bulk, no
// multicast) and streams right-operand CSs from HBM with 128-bit loads; every
// warp evaluates a whole tile of candidates per right row in registers.  A unary
// item applies every unary operator that reads the same source rows (~ X F G) to
// one load of each source chunk.  The fused epilogue per candidate is:
// fingerprint (warp reduce-scatter), acceptance (redux.sync over the positive-miss
// and negative-hit masks of bit 0), exact uniqueness in an open-addressing HBM
// hash set (claim by CAS, write the row, publish; a fingerprint match is verified
// word by word against the stored row), and per-level row statistics for the
// learned block order.  The last CTA of a launch writes the level's summary into
// the host's mapped ring.
//
// Semantics follow MojtabaValizadeh/ltl-learning-on-gpus, code/ltli6463.cu:
//   operators .......... :203-204 (~), :295 (&), :385 (|), :468 (X), :551-556 (F),
//                        :638-645 (G), :739-771 (U, both orders from one pair)
//   acceptance ......... :240-243 (positives need bit 0 set, negatives clear)
//   uniqueness ......... :224-231 (a candidate is stored iff its key is new)
//   relaxed keys ....... :57-141 (KEY_REF, types 1/2/3 and the exact 126-bit pack)
//   found .............. :243 (atomicCAS on a found word)
// Every device wait is bounded; giving up sets a status bit the host reads.
#include <atomic>

#include "ltl_kernels.cuh"

namespace ltlg {

namespace {

constexpr u64 WEYL = 0x9E3779B97F4A7C15ull;
constexpr u64 LENMASK = 0x7FFFFFFFFFFFFFFFull;
constexpr u64 M63 = 0x7FFFFFFFFFFFFFFFull;
constexpr u32 FIELD_PENDING = 0xFFFFFFFFu;
constexpr u32 FIELD_OVERFLOW = 0xFFFFFFFEu;
constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr long long MBAR_SPINS = 1ll << 24;    // bulk-copy completion wait

// MurmurHash3's 64-bit finaliser (Appleby, public domain).
__device__ __forceinline__ u64 fmix64(u64 x) {
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

// Operator classes: each kernel runs one class; within the unary class (~ X F G) and the
// and/or class the operator is a warp-uniform runtime value.
constexpr int OP_ANDOR = 8, OP_UNARY = 9;

template <int OP>
__device__ __forceinline__ u64 uop(u64 w, u64 meta, int rop) {
    const int op = OP == OP_UNARY ? rop : OP;
    const u64 m = meta & LENMASK;
    if (op == OP_NEG) return ~w & m;
    if (op == OP_X) return w >> 1;
    if (op == OP_F) return fin_bits(w);
    return glob_bits(w, m);  // OP_G
}

template <int OP>
__device__ __forceinline__ u64 bop(u64 a, u64 b, int rop) {
    const int op = OP == OP_ANDOR ? rop : OP;
    if (op == OP_AND) return a & b;
    if (op == OP_OR) return a | b;
    return until_bits(a, b);
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
// Bit 0 disagrees with the label (positives need 1, negatives 0); padding words are 0 with label 0.
// Acceptance at position 0, per pair of words: a positive trace where it fails (pmiss) or a
// negative trace (padding words count as negative) where it holds (nhit).
__device__ __forceinline__ u32 pmiss(u64 w0, u64 w1, u64 m0, u64 m1) {
    return (u32)(((~w0 & (m0 >> 63)) | (~w1 & (m1 >> 63))) & 1ull);
}
__device__ __forceinline__ u32 nhit(u64 w0, u64 w1, u64 m0, u64 m1) {
    return (u32)(((w0 & ~(m0 >> 63)) | (w1 & ~(m1 >> 63))) & 1ull);
}

__device__ __forceinline__ u64 ld_acquire(const u64 *p) {
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(u64 *p, u64 v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ u64 ld_volatile(const u64 *p) { return *(const volatile u64 *)p; }

// ---------------------------------------------------------------- mbarrier + bulk copy
__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
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
__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(u64 *bar, u32 parity) {
    for (long long i = 0; i < MBAR_SPINS; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
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
        constexpr int dummy = 0;
        (void)dummy;
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

// ---------------------------------------------------------------- candidate generators
// pre(c) loads the operand chunk every candidate of the batch shares (binary: the right
// row; unary: the word metadata); word(t, c, pre) gives words 2c, 2c+1 of candidate t.
template <int OP>
struct BinGen {
    const ulonglong2 *left;   // shared-memory tile, row stride nch
    const ulonglong2 *right;  // global right row
    int nch;
    int rop;
    __device__ __forceinline__ ulonglong2 pre(int c) const { return __ldg(right + c); }
    __device__ __forceinline__ ulonglong2 word(int t, int c, ulonglong2 r) const {
        if (OP == OP_U) {
            const ulonglong2 l = left[(t >> 1) * nch + c];
            const u64 lx = rev62(l.x), ly = rev62(l.y), rx = rev62(r.x), ry = rev62(r.y);
            if (t & 1) return make_ulonglong2(until_rev(lx | rx, lx), until_rev(ly | ry, ly));
            return make_ulonglong2(until_rev(lx | rx, rx), until_rev(ly | ry, ry));
        }
        const ulonglong2 l = left[t * nch + c];
        return make_ulonglong2(bop<OP>(l.x, r.x, rop), bop<OP>(l.y, r.y, rop));
    }
};

template <int OP>
struct UnGen {
    const u64 *src0;  // first source row of the group; rows are consecutive
    const ulonglong2 *meta;
    int pitch;
    int rop;
    __device__ __forceinline__ ulonglong2 pre(int c) const { return __ldg(meta + c); }
    __device__ __forceinline__ ulonglong2 word(int t, int c, ulonglong2 m) const {
        const ulonglong2 s = __ldg(reinterpret_cast<const ulonglong2 *>(src0 + (size_t)t * pitch) + c);
        return make_ulonglong2(uop<OP>(s.x, m.x, rop), uop<OP>(s.y, m.y, rop));
    }
};

// A stored row as its own candidate (letters).
struct RowGen {
    const ulonglong2 *r;
    __device__ __forceinline__ ulonglong2 pre(int c) const { return r[c]; }
    __device__ __forceinline__ ulonglong2 word(int, int, ulonglong2 p) const { return p; }
};

// Relaxed key of candidate t (KEY_REF), warp-cooperative; result valid in every lane.
template <class Gen>
__device__ void ref_key(const LevelArgs &A, const Gen &g, int t, int lane, u64 &kh, u64 &kl) {
    const int nch = A.pitch >> 1;
    u64 h = 0, l = 0;
    for (int c = lane; c < nch; c += 32) {
        const ulonglong2 w2 = g.word(t, c, g.pre(c));
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int i = 2 * c + e;
            if (i >= A.n) break;
            const u64 w = e ? w2.y : w2.x;
            if (A.rlx_type == 3) {
                // splitmix64 finaliser per word, folded by halves (ltli6463.cu:108-119)
                u64 x = w;
                x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
                x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
                x = x ^ (x >> 31);
                if (i < A.n / 2)
                    h ^= x;
                else
                    l ^= x;
            } else {
                const u32 km = A.kmeta[i];
                const u32 start = km & 0xFFFFu, count = (km >> 16) & 0xFFu, step = km >> 24;
                if (start >= 126 || count == 0) continue;
                u64 bits;
                if (step <= 1) {
                    bits = count >= 64 ? w : (w & ((1ull << count) - 1));
                } else {
                    bits = 0;
                    for (u32 q = 0; q < count; ++q) bits |= ((w >> (q * step)) & 1ull) << q;
                }
                const unsigned __int128 v = (unsigned __int128)bits << start;
                l |= (u64)v & M63;
                h |= (u64)(v >> 63) & M63;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const u64 ho = __shfl_xor_sync(FULL, h, o), lo = __shfl_xor_sync(FULL, l, o);
        if (A.rlx_type == 3) {
            h ^= ho;
            l ^= lo;
        } else {
            h |= ho;
            l |= lo;
        }
    }
    kh = h;
    kl = l;
}

// ---------------------------------------------------------------- uniqueness
enum { S_DONE = 0, S_PROBE = 1, S_CLAIM = 2, S_WAIT = 3, S_VERIFY = 4 };

__device__ __forceinline__ bool slot_free(u64 v, u32 gen) { return v == 0 || (u32)((v >> 32) & 0xFFu) != gen; }

// Per-level counts of stored rows by how they behave at position 0 (the acceptance bit):
// [0] holds on every positive trace, [1] holds on no negative trace.  Masks: bit l set when
// candidate l fails on some positive (pmiss) / holds on some negative (nhit).
__device__ __forceinline__ void count_row_stats(u64 *cnt, bool stored, u32 pmiss, u32 nhit, int lane) {
    const u32 bt = 1u << lane;
    const u32 k0 = __ballot_sync(FULL, stored && !(pmiss & bt)), k1 = __ballot_sync(FULL, stored && !(nhit & bt));
    if (lane == 0) {
        if (k0) atomicAdd(cnt + 0, (u64)__popc(k0));
        if (k1) atomicAdd(cnt + 1, (u64)__popc(k1));
    }
}

// Lane t owns candidate t (t < NC).  Every phase that touches whole CSs (writing the
// claimed rows, verifying fingerprint matches) is one chunk-major sweep over all the
// candidates concerned, so their loads are in flight together.  Claims are written and
// published before any lane waits on another warp's publication, so waits cannot cycle.
template <int NC, class Gen>
__device__ void resolve(const LevelArgs &A, const Gen &g, u64 fp, bool active, u64 parent, u64 kh, u64 kl,
                        u32 anyp, u32 anyn, int lane) {
    int state = active ? S_PROBE : S_DONE;
    const u64 tagbits = (fp >> 40) << 40;
    const u64 genbits = (u64)A.gen << 32;
    const u64 want = tagbits | genbits | FIELD_PENDING;
    u64 idx = fp & A.slot_mask;
    long long vrow = -1;
    u64 probes = 0;
    const int nch = A.pitch >> 1;
    while (__any_sync(FULL, state != S_DONE)) {
        if (state == S_PROBE) {
            for (;;) {
                u64 *sp = A.slots + idx;
                // CAS first: an empty slot is claimed in one round trip; otherwise the
                // returned value is the slot's content.
                u64 v = atomicCAS(sp, 0ull, want);
                if (v == 0ull) {
                    state = S_CLAIM;
                    break;
                }
                if (slot_free(v, A.gen)) {  // a slot of an older generation
                    const u64 old = atomicCAS(sp, v, want);
                    if (old == v) {
                        state = S_CLAIM;
                        break;
                    }
                    v = old;
                    if (slot_free(v, A.gen)) continue;
                }
                if ((v >> 40) == (tagbits >> 40)) {
                    const u32 f = (u32)v;
                    if (f == FIELD_PENDING) {
                        state = S_WAIT;
                        break;
                    }
                    if (f == FIELD_OVERFLOW) {
                        state = S_DONE;
                        break;
                    }
                    vrow = (long long)f - 1;
                    state = S_VERIFY;
                    break;
                }
                idx = (idx + 1) & A.slot_mask;
                if (++probes > A.slot_mask) {
                    atomicOr(&A.ctl->status, ST_TABLE);
                    state = S_DONE;
                    break;
                }
            }
        }
        // Claims: one row reservation per warp, one sweep writing every claimed CS, publish.
        const u32 cm = __ballot_sync(FULL, state == S_CLAIM);
        if (cm) {
            const int leader = __ffs(cm) - 1;
            u64 base = 0;
            if (lane == leader) base = atomicAdd(&A.ctl->row_count, (u64)__popc(cm));
            base = __shfl_sync(FULL, base, leader);
            const u64 cap = (u64)A.cap_rows;
#pragma unroll 2
            for (int c = lane; c < nch; c += 32) {
                const ulonglong2 p = g.pre(c);
#pragma unroll
                for (int t = 0; t < NC; ++t) {
                    if ((cm >> t) & 1u) {
                        const u64 row = base + __popc(cm & ((1u << t) - 1u));
                        if (row < cap) reinterpret_cast<ulonglong2 *>(A.cache + row * (u64)A.pitch)[c] = g.word(t, c, p);
                    }
                }
            }
            const u64 myrow = base + __popc(cm & ((1u << lane) - 1u));
            if (A.lstats && A.cost <= MAX_COSTS)
                count_row_stats(A.lstats + (u64)A.cost * LSTATS, state == S_CLAIM && myrow < cap, anyp, anyn, lane);
            if (state == S_CLAIM && myrow < cap) {
                A.parents[myrow] = parent;
                if (A.keys) {
                    A.keys[2 * myrow] = kh;
                    A.keys[2 * myrow + 1] = kl;
                }
            }
            __threadfence();
            __syncwarp();
            if (state == S_CLAIM) {
                u32 f = FIELD_OVERFLOW;
                if (myrow < cap)
                    f = (u32)(myrow + 1);
                else if ((atomicOr(&A.ctl->status, ST_OVERFLOW) & ST_OVERFLOW) == 0u)
                    atomicCAS(&A.ctl->overflow_cost, 0u, (u32)A.cost);
                st_release(A.slots + idx, tagbits | genbits | f);
                state = S_DONE;
            }
        }
        // Waits on other warps' publications (bounded).
        if (state == S_WAIT) {
            u32 f = FIELD_PENDING;
            for (long long s = 0; s < A.wait_spins; ++s) {
                f = (u32)ld_acquire(A.slots + idx);
                if (f != FIELD_PENDING) break;
                __nanosleep(128);
            }
            if (f == FIELD_PENDING) {
                atomicOr(&A.ctl->status, ST_WAIT);
                state = S_DONE;
            } else if (f == FIELD_OVERFLOW) {
                state = S_DONE;
            } else {
                vrow = (long long)f - 1;
                state = S_VERIFY;
            }
        }
        // Verification of fingerprint matches: one sweep comparing every candidate with its row.
        if (A.key_mode == KEY_EXACT) {
            const u32 vm = __ballot_sync(FULL, state == S_VERIFY);
            if (vm) {
                u32 vr[NC];
#pragma unroll
                for (int t = 0; t < NC; ++t) vr[t] = (u32)__shfl_sync(FULL, (u32)vrow, t);
                u32 diff = 0;
#pragma unroll 2
                for (int c = lane; c < nch; c += 32) {
                    const ulonglong2 p = g.pre(c);
#pragma unroll
                    for (int t = 0; t < NC; ++t) {
                        if ((vm >> t) & 1u) {
                            const ulonglong2 a = g.word(t, c, p);
                            const ulonglong2 b = __ldcg(reinterpret_cast<const ulonglong2 *>(
                                                            A.cache + (u64)vr[t] * (u64)A.pitch) + c);
                            diff |= (u32)((a.x != b.x) | (a.y != b.y)) << t;
                        }
                    }
                }
                const u32 anydiff = __reduce_or_sync(FULL, diff);
                if (state == S_VERIFY) {
                    if ((anydiff >> lane) & 1u) {
                        state = S_PROBE;
                        idx = (idx + 1) & A.slot_mask;
                    } else {
                        state = S_DONE;
                    }
                }
            }
        } else if (state == S_VERIFY) {
            const u64 eh = __ldcg(A.keys + 2 * vrow), el = __ldcg(A.keys + 2 * vrow + 1);
            if (eh == kh && el == kl) {
                state = S_DONE;
            } else {
                state = S_PROBE;
                idx = (idx + 1) & A.slot_mask;
            }
        }
    }
}

// Fingerprints, acceptance, found flag, uniqueness for NC candidates of one warp.
template <int NC, class Gen, class ParentOf>
__device__ __forceinline__ void finish(const LevelArgs &A, const Gen &g, u64 (&h)[NC], u32 bp, u32 bn, u32 valid,
                                       ParentOf parent_of, int lane) {
    const u64 sum = reduce_to_lane<NC>(h, lane);
    const u32 anyp = __reduce_or_sync(FULL, bp), anyn = __reduce_or_sync(FULL, bn);
    const u32 acc = ~(anyp | anyn) & valid;
    const u64 myparent = parent_of(lane);
    if (acc) {
        const int t = __ffs(acc) - 1;
        const u64 p = __shfl_sync(FULL, myparent, t);
        if (lane == 0 && atomicCAS(&A.ctl->found, 0ull, (1ull << 63) | p) == 0ull) A.ctl->found_cost = (u32)A.cost;
        if (A.stop_at_found) return;
    }
    if (A.check_only) return;
    u64 fp = fmix64(sum), kh = 0, kl = 0;
    if (A.key_mode == KEY_HASH64) {
        kh = fp;
    } else if (A.key_mode == KEY_REF) {
        for (int t = 0; t < NC; ++t) {
            if (!((valid >> t) & 1u)) continue;
            u64 a, b;
            ref_key(A, g, t, lane, a, b);
            if (lane == t) {
                kh = a;
                kl = b;
            }
        }
        fp = fmix64(kh ^ fmix64(kl + 0x5ad0dedull));
    }
    resolve<NC>(A, g, fp, (valid >> lane) & 1u, myparent, kh, kl, anyp, anyn, lane);
}

__device__ __forceinline__ bool found_stop(const LevelArgs &A) {
    return A.stop_at_found && ld_volatile(&A.ctl->found) != 0ull;
}

// ---------------------------------------------------------------- work items
// Operator of slot j of a fused unary block: 0 ~, 1 X, 2 F, 3 G.
__device__ __forceinline__ int unary_slot_op(int j) { return j == 0 ? OP_NEG : j == 1 ? OP_X : j == 2 ? OP_F : OP_G; }

// Candidate t of a fused unary item: source row t >> 2, operator slot t & 3.
struct FusedUnGen {
    const u64 *src0;  // first source row of the item; rows are consecutive
    const ulonglong2 *meta;
    int pitch;
    __device__ __forceinline__ ulonglong2 pre(int c) const { return __ldg(meta + c); }
    __device__ __forceinline__ ulonglong2 word(int t, int c, ulonglong2 m) const {
        const ulonglong2 s = __ldg(reinterpret_cast<const ulonglong2 *>(src0 + (size_t)(t >> 2) * pitch) + c);
        const int op = unary_slot_op(t & 3);
        return make_ulonglong2(uop<OP_UNARY>(s.x, m.x, op), uop<OP_UNARY>(s.y, m.y, op));
    }
};

// One warp evaluates every operator of `mask` on source rows [s, s + rows) (rows <=
// UNARY_ROWS): each source chunk is loaded once for all of them.
template <int HK>
__device__ __forceinline__ void unary_fused(const LevelArgs &A, int mask, long long s, int rows, int lane,
                                            u64 &evals) {
    constexpr int NC = 4 * UNARY_ROWS;
    const int nch = A.pitch >> 1;
    const ulonglong2 *meta = reinterpret_cast<const ulonglong2 *>(A.wmeta);
    const u64 *src0 = A.cache + (u64)s * A.pitch;
    u64 h[NC];
#pragma unroll
    for (int t = 0; t < NC; ++t) h[t] = 0;
    u32 bp = 0, bn = 0;
    for (int c0 = lane; c0 < nch; c0 += 64) {
        ulonglong2 sv[2][UNARY_ROWS], mv[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + 32 * u;
            if (c < nch) {
                mv[u] = __ldg(meta + c);
#pragma unroll
                for (int r = 0; r < UNARY_ROWS; ++r)
                    if (r < rows) sv[u][r] = __ldg(reinterpret_cast<const ulonglong2 *>(src0 + (size_t)r * A.pitch) + c);
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = c0 + 32 * u;
            if (c < nch) {
                const u64 k = (2ull * (u64)c + 1ull) * WEYL;
                const bool v0 = 2 * c < A.n, v1 = 2 * c + 1 < A.n;
                const ulonglong2 m = mv[u];
#pragma unroll
                for (int r = 0; r < UNARY_ROWS; ++r) {
                    if (r < rows) {
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            if ((mask >> j) & 1) {
                                const int op = unary_slot_op(j);
                                const u64 w0 = uop<OP_UNARY>(sv[u][r].x, m.x, op), w1 = uop<OP_UNARY>(sv[u][r].y, m.y, op);
                                h[4 * r + j] += hw<HK>(w0, k, v0) + hw<HK>(w1, k + WEYL, v1);
                                bp |= pmiss(w0, w1, m.x, m.y) << (4 * r + j);
                                bn |= nhit(w0, w1, m.x, m.y) << (4 * r + j);
                            }
                        }
                    }
                }
            }
        }
    }
    u32 valid = 0;
    for (int r = 0; r < rows; ++r) valid |= (u32)(mask & 15) << (4 * r);
    FusedUnGen g{src0, meta, A.pitch};
    finish<NC>(A, g, h, bp, bn, valid,
               [&](int t) { return pack_parent(unary_slot_op(t & 3), (u64)(s + (t >> 2)), 0); }, lane);
    evals += (u64)__popc(valid);
}

template <int OP, int TL, int HK>
__device__ void binary_row(const LevelArgs &A, int rop, const ulonglong2 *tile, int nl, long long l_first,
                           long long r, int lane, u64 &evals) {
    constexpr int NC = OP == OP_U ? 2 * TL : TL;
    const int nch = A.pitch >> 1;
    const ulonglong2 *R = reinterpret_cast<const ulonglong2 *>(A.cache + (u64)r * A.pitch);
    const ulonglong2 *meta = reinterpret_cast<const ulonglong2 *>(A.wmeta);
    u64 h[NC];
#pragma unroll
    for (int t = 0; t < NC; ++t) h[t] = 0;
    u32 bp = 0, bn = 0;
    for (int c0 = lane; c0 < nch; c0 += 128) {
        ulonglong2 rvv[4], mv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u;
            if (c < nch) {
                rvv[u] = __ldg(R + c);
                mv[u] = __ldg(meta + c);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + 32 * u;
            if (c >= nch) continue;
            const u64 k = (2ull * (u64)c + 1ull) * WEYL;
            const ulonglong2 rv = rvv[u], m = mv[u];
            const bool v0 = 2 * c < A.n, v1 = 2 * c + 1 < A.n;
            const u64 rx = OP == OP_U ? rev62(rv.x) : 0ull, ry = OP == OP_U ? rev62(rv.y) : 0ull;
#pragma unroll
            for (int t = 0; t < TL; ++t) {
                if (t < nl) {
                    const ulonglong2 lv = tile[t * nch + c];
                    if (OP == OP_U) {
                        const u64 lx = rev62(lv.x), ly = rev62(lv.y);
                        const u64 ax = lx | rx, ay = ly | ry;
                        const u64 a0 = until_rev(ax, rx), a1 = until_rev(ay, ry);  // l U r
                        const u64 b0 = until_rev(ax, lx), b1 = until_rev(ay, ly);  // r U l
                        h[2 * t] += hw<HK>(a0, k, v0) + hw<HK>(a1, k + WEYL, v1);
                        h[2 * t + 1] += hw<HK>(b0, k, v0) + hw<HK>(b1, k + WEYL, v1);
                        bp |= (pmiss(a0, a1, m.x, m.y) << (2 * t)) | (pmiss(b0, b1, m.x, m.y) << (2 * t + 1));
                        bn |= (nhit(a0, a1, m.x, m.y) << (2 * t)) | (nhit(b0, b1, m.x, m.y) << (2 * t + 1));
                    } else {
                        const u64 w0 = bop<OP>(lv.x, rv.x, rop), w1 = bop<OP>(lv.y, rv.y, rop);
                        h[t] += hw<HK>(w0, k, v0) + hw<HK>(w1, k + WEYL, v1);
                        bp |= pmiss(w0, w1, m.x, m.y) << t;
                        bn |= nhit(w0, w1, m.x, m.y) << t;
                    }
                }
            }
        }
    }
    const int cnt = OP == OP_U ? 2 * nl : nl;
    const u32 valid = cnt >= 32 ? FULL : ((1u << cnt) - 1u);
    BinGen<OP> g{tile, R, nch, rop};
    const int op = OP == OP_ANDOR ? rop : OP;
    finish<NC>(A, g, h, bp, bn, valid,
               [&](int t) {
                   if (OP == OP_U) {
                       const u64 l = (u64)(l_first + (t >> 1));
                       return (t & 1) ? pack_parent(op, (u64)r, l) : pack_parent(op, l, (u64)r);
                   }
                   return pack_parent(op, (u64)(l_first + t), (u64)r);
               },
               lane);
    evals += (u64)cnt;
}

template <int OP, int TL, int HK>
__device__ __noinline__ bool binary_item(const LevelArgs &A, int rop, const BlockDesc &B, long long local, u64 *tile,
                                            u64 *bar, u32 &phase, unsigned *next_row, int lane, u64 &evals) {
    constexpr int TLOP = OP == OP_U ? TL / 2 : TL;  // U makes two candidates per pair
    const long long tl = local / B.tiles_r, tr = local % B.tiles_r;
    const long long l_first = B.l0 + tl * TLOP;
    const int nl = (int)min((long long)TLOP, B.l1 - l_first);
    const long long r_first = B.r0 + tr * A.right_chunk;
    const long long r_end = min(B.r1, r_first + (long long)A.right_chunk);
    if (threadIdx.x == 0) {
        fence_proxy_async();
        const u32 bytes = (u32)nl * (u32)A.pitch * 8u;
        mbar_expect_tx(bar, bytes);
        bulk_g2s(tile, A.cache + (u64)l_first * A.pitch, bytes, bar);
    }
    const bool ok = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(&A.ctl->status, ST_TMA);
        mbar_wait_bounded(bar, phase);  // let the copy in flight land before the CTA leaves
        return false;
    }
    phase ^= 1u;
    const ulonglong2 *t2 = reinterpret_cast<const ulonglong2 *>(tile);
    // warps take the item's right rows one at a time (less waiting at the item's end)
    for (;;) {
        long long r = 0;
        if (lane == 0) r = r_first + (long long)atomicAdd(next_row, 1u);
        r = __shfl_sync(FULL, r, 0);
        if (r >= r_end) break;
        if (__any_sync(FULL, found_stop(A))) break;  // warp-uniform: lanes must not split
        binary_row<OP, TLOP, HK>(A, rop, t2, nl, l_first, r, lane, evals);
    }
    return true;
}

// The unary part of a level: fused blocks (every unary operator over the same source rows),
// items of A.unary_rows source rows; the CTA's warps take UNARY_ROWS rows at a time.
template <int HK>
__device__ __noinline__ void unary_item(const LevelArgs &A, const BlockDesc &B, long long local, int warp, int nwarps,
                                        int lane, u64 &evals) {
    const long long s_first = B.r0 + local * A.unary_rows;
    const long long s_end = min(B.r1, s_first + (long long)A.unary_rows);
    for (long long s = s_first + (long long)warp * UNARY_ROWS; s < s_end; s += (long long)nwarps * UNARY_ROWS) {
        if (__any_sync(FULL, found_stop(A))) return;  // warp-uniform: lanes must not split
        unary_fused<HK>(A, B.opmask, s, (int)min((long long)UNARY_ROWS, s_end - s), lane, evals);
    }
}

// Copy the arguments and the level's plan header into shared memory (thread 0).
__device__ __forceinline__ void load_level(LevelArgs &A, const LevelArgs *A0) {
    A = *A0;
    const DevLevel *L = A.lev;
    A.cost = L->cost;
    A.check_only = L->check_only;
    A.right_chunk = L->right_chunk;
    A.unary_rows = L->unary_rows;
}

// The end of a level-kernel launch: the last CTA to finish resets the CTA count and, when
// the host keeps a ring of level summaries in mapped memory, writes the control block and
// the plan header into the level's slot, so the host reads them without a copy on the
// stream.  No CTA waits for another.
__device__ __forceinline__ void level_summary(const LevelArgs &A) {
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const u32 done = atomicAdd(&A.ctl->ctas_done, 1u);
        s_last = done == gridDim.x - 1 ? 1 : 0;
        if (s_last) A.ctl->ctas_done = 0u;
    }
    __syncthreads();
    if (!s_last || !A.ring) return;
    __threadfence();
    constexpr int CW = sizeof(DevCtl) / 8, LW = offsetof(DevLevel, blocks) / 8;
    const int R = A.ring_slots;
    const int slot = ((A.lev->seq - 1) % R + R) % R;
    u64 *dc = reinterpret_cast<u64 *>(A.ring) + (u64)slot * CW;
    u64 *dl = reinterpret_cast<u64 *>(reinterpret_cast<char *>(A.ring) + (u64)R * sizeof(DevCtl) +
                                      (u64)slot * sizeof(DevLevel));
    const u64 *sc = reinterpret_cast<const u64 *>(A.ctl), *sl = reinterpret_cast<const u64 *>(A.lev);
    for (int i = threadIdx.x; i < CW + LW; i += blockDim.x) {
        if (i < CW)
            dc[i] = ld_volatile(sc + i);
        else
            dl[i - CW] = ld_volatile(sl + (i - CW));
    }
    __threadfence_system();
}

// Leading entries of the item table kept in shared memory (read once per item in a learned
// order).  Small enough that three CTAs with a 64 KB tile still fit the 196 KB carveout.
constexpr int RANGE_CACHE = 32;

__device__ __forceinline__ int find_block(const BlockDesc *blocks, int nb, long long in_op) {
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blocks[mid].item0 <= in_op)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One level: every work item of the plan in A.lev, drained through one queue
// (ctl->queue[0] up to lev->items_end).  Items are numbered in the plain order: the unary
// blocks' items, then the & blocks', the | blocks', the U blocks'.  Under a learned order the
// queue runs through the item table instead and thread 0 maps each claimed item to its plain
// number.  A unary item is A.unary_rows source rows of a unary block (every operator of its
// mask on each row); a binary item stages a tile of left rows in shared memory with one bulk
// copy, and the CTA's warps take the item's right rows one at a time.
// Three CTAs per SM with an 8-row tile (64 KB of shared memory at n = 1000); four with a
// 4- or 2-row tile, which caps registers at 64 (measured faster end to end than 80 at three).
template <int TL, int HK>
__global__ void __launch_bounds__(256, TL <= 4 ? 4 : 3) level_kernel(const LevelArgs *__restrict__ A0) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    u64 *tile = reinterpret_cast<u64 *>(smem_raw);
    __shared__ __align__(16) LevelArgs A;
    __shared__ __align__(8) u64 bar;
    __shared__ ItemRange s_rng[RANGE_CACHE];
    __shared__ long long s_item, s_hi, s_ub[5], s_cls[4], s_and;
    __shared__ int s_halt, s_nub, s_nb[7], s_nr, s_learned;
    __shared__ unsigned s_next_row;
    __shared__ u64 s_evals;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        load_level(A, A0);
        const DevLevel *L = A.lev;
        s_halt = L->halt;
        s_hi = L->items_end;
        s_nub = L->nublocks;
        long long b = 0;
        for (int k = 0; k < 4; ++k) {
            s_ub[k] = b;
            b += k < s_nub ? L->ublocks[k].items : 0;
        }
        s_ub[4] = b;
        s_cls[0] = 0;
        s_cls[1] = b;
        s_cls[2] = s_cls[1] + L->total_items[OP_AND] + L->total_items[OP_OR];
        s_cls[3] = s_cls[2] + L->total_items[OP_U];
        s_and = L->total_items[OP_AND];
        for (int op = 0; op < 7; ++op) s_nb[op] = L->nblocks[op];
        s_nr = L->nranges;
        s_learned = L->learned_order;
        mbar_init(&bar, 1);
        fence_mbar_init();
        s_evals = 0;
    }
    __syncthreads();
    if (!s_halt && s_hi > 0) {
        if (s_learned) {
            for (int e = threadIdx.x; e < s_nr && e < RANGE_CACHE; e += blockDim.x) s_rng[e] = A.lev->ranges[e];
            __syncthreads();
        }
        u64 evals = 0;
        u32 phase = 0;
        int cur = 0;  // thread 0, learned order: table entry of the last item (claimed in increasing order)
        for (;;) {
            if (threadIdx.x == 0) {
                long long it = -1;
                if (!found_stop(A)) {
                    it = (long long)atomicAdd(&A.ctl->queue[0], 1ull);
                    if (it >= s_hi) it = -1;
                }
                if (it >= 0 && s_learned) {  // the entry holding the item: the last one with item0 <= it
                    const ItemRange *rng = A.lev->ranges;
                    auto item0_of = [&](int e) { return e < RANGE_CACHE ? s_rng[e].item0 : rng[e].item0; };
                    while (cur + 1 < s_nr && item0_of(cur + 1) <= it) ++cur;
                    const ItemRange R = cur < RANGE_CACHE ? s_rng[cur] : rng[cur];
                    it = R.plain0 + (it - R.item0);
                }
                s_item = it;
                s_next_row = 0;
            }
            __syncthreads();
            const long long item = s_item;
            if (item < 0) break;
            bool ok = true;
            if (item < s_cls[1]) {
                int k = 0;
                while (k < s_nub - 1 && item >= s_ub[k + 1]) ++k;
                unary_item<HK>(A, A.lev->ublocks[k], item - s_ub[k], warp, nwarps, lane, evals);
            } else if (item < s_cls[2]) {
                const long long in_cls = item - s_cls[1];
                const int op = in_cls < s_and ? OP_AND : OP_OR;
                const long long in_op = op == OP_AND ? in_cls : in_cls - s_and;
                const BlockDesc *blocks = A.lev->blocks[op];
                const BlockDesc B = blocks[find_block(blocks, s_nb[op], in_op)];
                ok = binary_item<OP_ANDOR, TL, HK>(A, op, B, in_op - B.item0, tile, &bar, phase, &s_next_row, lane, evals);
            } else {
                const long long in_op = item - s_cls[2];
                const BlockDesc *blocks = A.lev->blocks[OP_U];
                const BlockDesc B = blocks[find_block(blocks, s_nb[OP_U], in_op)];
                ok = binary_item<OP_U, TL, HK>(A, OP_U, B, in_op - B.item0, tile, &bar, phase, &s_next_row, lane, evals);
            }
            if (!ok) break;
            __syncthreads();  // every warp is done with the tile before the next copy
        }
        if (lane == 0 && evals) atomicAdd(&s_evals, evals);
        __syncthreads();
        if (threadIdx.x == 0 && s_evals) atomicAdd(&A.ctl->evaluated, s_evals);
    }
    level_summary(A);
}

// Letters: register rows [0, nalpha) in the hash set (duplicate letters stay rows,
// as the reference stores every letter, ltli6463.cu:1134, :1189-1190).  One warp.
template <int HK>
__global__ void insert_letters_kernel(const LevelArgs *__restrict__ pA, int nalpha) {
    const LevelArgs &A = *pA;
    const int lane = threadIdx.x & 31, j = threadIdx.x >> 5;  // warp j: letter j
    const int nch = A.pitch >> 1;
    const ulonglong2 *meta = reinterpret_cast<const ulonglong2 *>(A.wmeta);
    const bool mine = j < nalpha;
    const u64 *row = A.cache + (u64)(mine ? j : 0) * A.pitch;
    const RowGen g{reinterpret_cast<const ulonglong2 *>(row)};
    u64 fp = 0, kh = 0, kl = 0;
    if (mine) {  // the letters' fingerprints and statistics, all letters at once
        u64 h[1] = {0};
        u32 pm = 0, nh = 0;  // position 0: fails on a positive / holds on a negative
#pragma unroll 4
        for (int c = lane; c < nch; c += 32) {
            const u64 k = (2ull * (u64)c + 1ull) * WEYL;
            const ulonglong2 w = reinterpret_cast<const ulonglong2 *>(row)[c];
            h[0] += hw<HK>(w.x, k, 2 * c < A.n) + hw<HK>(w.y, k + WEYL, 2 * c + 1 < A.n);
            const ulonglong2 m = meta[c];
            pm |= pmiss(w.x, w.y, m.x, m.y);
            nh |= nhit(w.x, w.y, m.x, m.y);
        }
        if (A.lstats && A.cf[0] <= MAX_COSTS)  // every letter is a stored row of the letter level
            count_row_stats(A.lstats + (u64)A.cf[0] * LSTATS, lane == 0, __any_sync(FULL, pm) ? 1u : 0u,
                            __any_sync(FULL, nh) ? 1u : 0u, lane);
        const u64 sum = reduce_to_lane<1>(h, lane);
        fp = fmix64(sum);
        if (A.key_mode == KEY_HASH64) {
            kh = fp;
        } else if (A.key_mode == KEY_REF) {
            ref_key(A, g, 0, lane, kh, kl);
            fp = fmix64(kh ^ fmix64(kl + 0x5ad0dedull));
        }
    }
    // Registration in letter order, one warp at a time (a duplicate letter stays a row but
    // the set keeps the first one, as the reference's sequential inserts do).
    for (int turn = 0; turn < nalpha; ++turn) {
        if (turn == j) {
            // Probe with lane 0; a fingerprint match is verified by the whole warp.
            const u64 tagbits = (fp >> 40) << 40, genbits = (u64)A.gen << 32;
            u64 idx = fp & A.slot_mask;
            for (u64 probe = 0; probe <= A.slot_mask; ++probe, idx = (idx + 1) & A.slot_mask) {
                u64 v = 0;
                int action = 0;  // 0 next, 1 claimed, 2 compare
                if (lane == 0) {
                    v = ld_acquire(A.slots + idx);
                    if (slot_free(v, A.gen)) {
                        const u64 old = atomicCAS(A.slots + idx, v, tagbits | genbits | (u64)(j + 1));
                        if (old == v) {
                            action = 1;
                        } else {
                            v = old;
                        }
                    }
                    if (action == 0 && (v >> 40) == (tagbits >> 40) && (u32)v < FIELD_OVERFLOW) action = 2;
                }
                action = __shfl_sync(FULL, action, 0);
                v = __shfl_sync(FULL, v, 0);
                if (action == 1) {
                    if (lane == 0) {
                        A.parents[j] = pack_parent(OP_ATOM, 0, 0);
                        if (A.keys) {
                            A.keys[2 * j] = kh;
                            A.keys[2 * j + 1] = kl;
                        }
                    }
                    break;
                }
                if (action == 2) {
                    const u64 other = (u64)(u32)v - 1;
                    bool same;
                    if (A.key_mode == KEY_EXACT) {
                        bool diff = false;
                        const ulonglong2 *ex = reinterpret_cast<const ulonglong2 *>(A.cache + other * A.pitch);
                        for (int c = lane; c < nch; c += 32) {
                            const ulonglong2 a = g.word(0, c, g.pre(c)), b = __ldcg(ex + c);
                            diff |= (a.x != b.x) | (a.y != b.y);
                        }
                        same = !__any_sync(FULL, diff);
                    } else {
                        same = A.keys[2 * other] == kh && A.keys[2 * other + 1] == kl;
                    }
                    if (same) {
                        if (lane == 0) A.parents[j] = pack_parent(OP_ATOM, 0, 0);
                        break;
                    }
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
}

// Tree of the found candidate: entries (row, parents) breadth first; entry 0 is the root
// (row ~0).  out[0] = entries written, out[1] = 1 when the buffer was too small.
__global__ void walk_kernel(const u64 *parents, int nalpha, u64 found, u64 *out, int cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    u64 *e = out + 2;
    int count = 0, head = 0, overflow = 0;
    e[0] = ~0ull;
    e[1] = found & ~(1ull << 63);
    count = 1;
    while (head < count) {
        const u64 p = e[2 * head + 1];
        const int op = parent_op(p);
        u64 kids[2] = {parent_left(p), parent_right(p)};
        const int nk = (op == OP_AND || op == OP_OR || op == OP_U) ? 2 : (op == OP_ATOM ? 0 : 1);
        for (int q = 0; q < nk; ++q) {
            if (kids[q] >= (u64)nalpha) {
                if (count >= cap) {
                    overflow = 1;
                    break;
                }
                e[2 * count] = kids[q];
                e[2 * count + 1] = parents[kids[q]];
                ++count;
            }
        }
        ++head;
    }
    out[0] = (u64)count;
    out[1] = (u64)overflow;
}

// Operator + fingerprint on independent rows, for kernel-level parity tests.  One warp per row.
__global__ void apply_op_kernel(int op, const u64 *a, const u64 *b, const u64 *wmeta, int n, int pitch, int count,
                                u64 *out, u64 *out2, u64 *fp) {
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= count) return;
    u64 h1 = 0, h2 = 0;
    for (int i = lane; i < pitch; i += 32) {
        const u64 x = a[(u64)row * pitch + i], y = b ? b[(u64)row * pitch + i] : 0;
        const u64 m = wmeta[i];
        u64 w = 0, w2 = 0;
        switch (op) {
        case OP_NEG: w = uop<OP_NEG>(x, m, OP_NEG); break;
        case OP_X: w = uop<OP_X>(x, m, OP_X); break;
        case OP_F: w = uop<OP_F>(x, m, OP_F); break;
        case OP_G: w = uop<OP_G>(x, m, OP_G); break;
        case OP_AND: w = bop<OP_AND>(x, y, OP_AND); break;
        case OP_OR: w = bop<OP_OR>(x, y, OP_OR); break;
        case OP_U:
            w = until_bits(x, y);
            w2 = until_bits(y, x);
            break;
        default: w = x; break;
        }
        out[(u64)row * pitch + i] = w;
        if (out2) out2[(u64)row * pitch + i] = w2;
        const u64 key = (u64)(i + 1) * WEYL;
        h1 += hw<1>(w, key, i < n);
        h2 += hw<1>(w2, key, i < n);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        h1 += __shfl_xor_sync(FULL, h1, o);
        h2 += __shfl_xor_sync(FULL, h2, o);
    }
    if (lane == 0) {
        fp[row] = fmix64(h1);
        if (out2) fp[count + row] = fmix64(h2);
    }
}

// A formula as a postfix program (op, arg) evaluated on every trace at once: thread t holds
// trace t's CS of each subformula on a stack in global memory laid out [depth][n], so
// neighbouring threads touch neighbouring words.  Letters read atoms[arg * n + t]; the
// operators are the enumerator's own (uop / bop / until_bits).
__global__ void eval_formula_kernel(const int *__restrict__ prog, int len, const u64 *__restrict__ atoms,
                                    const u64 *__restrict__ lenmask, int n, u64 *__restrict__ stack,
                                    u64 *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const u64 m = lenmask[t];
    int sp = 0;
    for (int k = 0; k < len; ++k) {
        const int op = prog[2 * k], arg = prog[2 * k + 1];
        u64 v;
        if (op == OP_ATOM) {
            v = atoms[(u64)arg * n + t];
        } else if (op == OP_NEG || op == OP_X || op == OP_F || op == OP_G) {
            v = uop<OP_UNARY>(stack[(u64)(sp - 1) * n + t], m, op);
            --sp;
        } else {
            const u64 y = stack[(u64)(sp - 1) * n + t], x = stack[(u64)(sp - 2) * n + t];
            v = op == OP_U ? until_bits(x, y) : bop<OP_ANDOR>(x, y, op);
            sp -= 2;
        }
        stack[(u64)sp * n + t] = v;
        ++sp;
    }
    out[t] = stack[t];
}

}  // namespace

cudaError_t launch_eval_formula(const int *prog, int len, const u64 *atoms, const u64 *lenmask, int n, u64 *stack,
                                u64 *out, cudaStream_t s) {
    eval_formula_kernel<<<(n + 127) / 128, 128, 0, s>>>(prog, len, atoms, lenmask, n, stack, out);
    return cudaGetLastError();
}

int level_kernel_smem_bytes(int left_tile, int pitch) { return left_tile * pitch * 8; }

// The dynamic shared-memory limit is a per-device function attribute: each device keeps the
// largest size enabled on it so far (0 = the 48 KiB default).
template <int TL, int HK>
static cudaError_t smem_attr(int smem) {
    constexpr int MAX_DEVICES = 64;
    static std::atomic<int> attr_set[MAX_DEVICES];
    if (smem <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < MAX_DEVICES && smem <= attr_set[dev].load()) return cudaSuccess;
    e = cudaFuncSetAttribute(level_kernel<TL, HK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess && dev >= 0 && dev < MAX_DEVICES) {
        int cur = attr_set[dev].load();
        while (cur < smem && !attr_set[dev].compare_exchange_weak(cur, smem)) {
        }
    }
    return e;
}

template <int TL, int HK>
static cudaError_t launch_tl(const LevelArgs &a, const LevelArgs *d, int grid, int block, cudaStream_t s) {
    const int smem = level_kernel_smem_bytes(TL, a.pitch);
    cudaError_t e = smem_attr<TL, HK>(smem);
    if (e != cudaSuccess) return e;
    level_kernel<TL, HK><<<grid, block, smem, s>>>(d);
    return cudaGetLastError();
}

template <int TL, int HK>
static int occupancy_tl(int block, int pitch) {
    const int smem = level_kernel_smem_bytes(TL, pitch);
    if (smem_attr<TL, HK>(smem) != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, level_kernel<TL, HK>, block, smem) == cudaSuccess ? n : 0;
}

cudaError_t launch_level(const LevelArgs &a, const LevelArgs *d, int grid, int block, cudaStream_t s) {
    if (a.hash_kind == 1)
        return a.left_tile == 2   ? launch_tl<2, 1>(a, d, grid, block, s)
               : a.left_tile == 4 ? launch_tl<4, 1>(a, d, grid, block, s)
                                  : launch_tl<8, 1>(a, d, grid, block, s);
    return a.left_tile == 2   ? launch_tl<2, 0>(a, d, grid, block, s)
           : a.left_tile == 4 ? launch_tl<4, 0>(a, d, grid, block, s)
                              : launch_tl<8, 0>(a, d, grid, block, s);
}

int level_kernel_max_ctas_per_sm(int left_tile, int hash_kind, int block, int pitch) {
    if (hash_kind == 1)
        return left_tile == 2   ? occupancy_tl<2, 1>(block, pitch)
               : left_tile == 4 ? occupancy_tl<4, 1>(block, pitch)
                                : occupancy_tl<8, 1>(block, pitch);
    return left_tile == 2   ? occupancy_tl<2, 0>(block, pitch)
           : left_tile == 4 ? occupancy_tl<4, 0>(block, pitch)
                            : occupancy_tl<8, 0>(block, pitch);
}

cudaError_t launch_insert_letters(const LevelArgs &a, const LevelArgs *d, int nalpha, cudaStream_t s) {
    if (a.hash_kind == 1)
        insert_letters_kernel<1><<<1, 32 * (nalpha > 0 ? nalpha : 1), 0, s>>>(d, nalpha);
    else
        insert_letters_kernel<0><<<1, 32 * (nalpha > 0 ? nalpha : 1), 0, s>>>(d, nalpha);
    return cudaGetLastError();
}

cudaError_t launch_walk(const u64 *parents, int nalpha, u64 found, u64 *out, int cap, cudaStream_t s) {
    walk_kernel<<<1, 32, 0, s>>>(parents, nalpha, found, out, cap);
    return cudaGetLastError();
}

cudaError_t launch_apply_op(int op, const u64 *a, const u64 *b, const u64 *wmeta, int n, int pitch, int count,
                            u64 *out, u64 *out2, u64 *fp, cudaStream_t s) {
    const int warps = 4;
    apply_op_kernel<<<(count + warps - 1) / warps, warps * 32, 0, s>>>(op, a, b, wmeta, n, pitch, count, out, out2,
                                                                       fp);
    return cudaGetLastError();
}

}  // namespace ltlg
