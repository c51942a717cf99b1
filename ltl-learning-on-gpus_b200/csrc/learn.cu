// The level kernel of the characteristic-set (CS) enumeration for sm_100a, and the planner
// that runs inside it.
//
// One CTA per SM, 32 warps.  Warp 0 is the producer: it takes work items from the instance's
// queue (a 64-bit counter tagged with the plan's sequence number), fills a ring of item slots
// in shared memory, stages each binary item's tile of left-operand CSs with one bulk copy
// (cp.async.bulk, no multicast, completion on the slot's mbarrier), and prefetches the item's
// right-operand (or unary source) rows into L2 with one bulk prefetch.  Warps 1..31 are
// consumers: they take the rows of the oldest slot one at a time, evaluate every candidate of
// a row in registers, and run the fused epilogue per candidate: fingerprint (warp
// reduce-scatter), acceptance (redux.sync over positive-miss / negative-hit bits of position
// 0), the find record, exact uniqueness in an open-addressing HBM hash set (claim by CAS,
// write the row, publish; a fingerprint match is verified word by word against the stored row,
// which is prefetched into L2 as soon as the match is seen), and per-level row statistics.
// A consumer leaves a slot through the slot's "empty" mbarrier, so no warp waits for another
// at item boundaries.
//
// The warp that finishes a level's last item closes the level (level start, the find) and
// plans the next level in the reference's block order, on the device; with `persist` the
// producers then take the next level's items in the same launch.  No CTA ever waits for a
// particular other CTA: a level ends when its items are done, whoever did them.
//
// The find follows the reference's order: the reference runs a level's blocks one after the
// other and stops after the first block that holds an accepting candidate
// (code/ltli6463.cu:1232-1234), so here the find is the accepting candidate of the smallest
// block position (an atomicMin on cost << 32 | position); items of later blocks are skipped once
// a find is known, items of earlier blocks still run.
//
// Semantics follow MojtabaValizadeh/ltl-learning-on-gpus, code/ltli6463.cu:
//   acceptance ......... :240-243 (positives need bit 0 set, negatives clear)
//   uniqueness ......... :224-231 (a candidate is stored iff its key is new)
//   relaxed keys ....... :57-141 (KEY_REF, types 1/2/3 and the exact 126-bit pack)
//   level / block order  :1199-1445 (NegType rule :1212)
// Every device wait is bounded; giving up sets a status bit the host reads.
#include <atomic>

#include "ltlgpu.h"
#include "ops.cuh"
#include "score.cuh"

namespace ltlg {

namespace {

constexpr int OP_ANDOR_CLASS = 8;              // binary_row's class of & and | (the operator is a runtime value)
constexpr int ENTRY_CACHE = 256;               // item starts of a plan's first entries kept in shared memory
constexpr int NWARPS = LEVEL_THREADS / 32;
constexpr int NCONS = NWARPS - 1;              // consumer warps per CTA
static_assert(NCONS == LEVEL_CONSUMERS, "consumer warps");
constexpr unsigned long long SPLIT_MAX_CANDS = 8192;  // levels below: rows split over warps (8k, 64k, 512k measured)
constexpr int WU = 1;  // chunks per lane loaded per round of a claim's write sweep (2 and 4 measured slower)

constexpr u64 PIPE_WAIT_NS = 30000000000ull;   // a consumer's wait for the producer (beyond every producer bound)
constexpr u64 EMPTY_WAIT_NS = 10000000000ull;  // the producer's wait for the consumers to leave a slot
constexpr u64 STALL_NS = 4000000000ull;        // no level progress while waiting for the next plan

// One work item in flight, written by the producer.
struct Slot {
    u64 full;                 // mbarrier: the producer filled the slot (and its tile landed)
    u64 empty;                // mbarrier: every consumer left the slot
    long long row0;           // binary: first right row; unary: first source row
    long long l_first;        // binary: first left row of the tile
    long long e_l0, e_r0, e_R;  // the entry's first left row, first right (source) row, right rows
    long long plan_items;     // items of the plan: the item done that brings `done` to it ends the level
    unsigned next_row;        // consumers take rows here
    unsigned rows_done;
    unsigned evals;           // candidates evaluated in this item
    int kind;                 // ENT_*; 0 = the producer has ended
    int op;                   // binary: OP_AND / OP_OR / OP_U; unary: opmask
    int nl;                   // binary: left rows in the tile
    int nrows;                // rows of the item
    int pos;                  // the entry's block position
    int upos[4];              // unary: block position of each slot operator
    int cost;
    int check_only;
    int stop;                 // remaining rows are skipped (a find at or before this entry)
    int inst;                 // the item's instance (index into Launch::args)
    int trace_first;          // the producer's first item of this plan (level stamps)
    int split;                // units per row: 1, or (a small level) one per left row / unary operator
    int units;                // nrows * split: what the consumers take
    int overflowed;           // the cache had overflowed when the item was claimed (or a claim here
                              // overflowed): the rows' new CSs take no hash slots
    InstArgs args;            // its arguments as they were when the item was claimed (a batch slot's
                              // arguments change when it takes the next instance)
};

// ---------------------------------------------------------------- candidate generators
// pre(c) loads everything of chunk c that the set's candidates read from global memory
// (binary: the right row; unary: the source row and the word metadata); word(t, c, pre) gives
// words 2c, 2c+1 of candidate t from it (and the shared-memory tile).  A sweep that stores
// words can so issue the loads of several chunks before its first store.
template <int OPC>
struct BinGen {
    using Pre = ulonglong2;
    const ulonglong2 *left;   // shared-memory tile, row stride nch
    const ulonglong2 *right;  // global right row
    int nch;
    int rop;
    __device__ __forceinline__ Pre pre(int c) const { return __ldcg(right + c); }
    __device__ __forceinline__ ulonglong2 word(int t, int c, ulonglong2 r) const {
        if (OPC == OP_U) {
            const ulonglong2 l = left[(t >> 1) * nch + c];
            const u64 lx = rev62(l.x), ly = rev62(l.y), rx = rev62(r.x), ry = rev62(r.y);
            if (t & 1) return make_ulonglong2(until_rev(lx | rx, lx), until_rev(ly | ry, ly));
            return make_ulonglong2(until_rev(lx | rx, rx), until_rev(ly | ry, ry));
        }
        const ulonglong2 l = left[t * nch + c];
        return rop == OP_AND ? make_ulonglong2(l.x & r.x, l.y & r.y) : make_ulonglong2(l.x | r.x, l.y | r.y);
    }
};

// Candidate t of a fused unary row: operator slot t (0 ~, 1 X, 2 F, 3 G) of one source row.
struct UnPre {
    ulonglong2 m, s;  // word metadata, source words
};
struct UnGen {
    using Pre = UnPre;
    const ulonglong2 *src;
    const ulonglong2 *meta;
    __device__ __forceinline__ Pre pre(int c) const { return UnPre{__ldcg(meta + c), __ldcg(src + c)}; }
    __device__ __forceinline__ ulonglong2 word(int t, int, const Pre &p) const {
        const int op = unary_slot_op(t);
        return make_ulonglong2(unary_word(op, p.s.x, p.m.x & LENMASK), unary_word(op, p.s.y, p.m.y & LENMASK));
    }
};

// A stored row as its own candidate (letters).
struct RowGen {
    using Pre = ulonglong2;
    const ulonglong2 *r;
    __device__ __forceinline__ ulonglong2 pre(int c) const { return r[c]; }
    __device__ __forceinline__ ulonglong2 word(int, int, ulonglong2 p) const { return p; }
};

// Relaxed key of candidate t (KEY_REF), warp-cooperative; result valid in every lane.
template <class Gen>
__device__ void ref_key(const InstArgs &A, const Gen &g, int t, int lane, u64 &kh, u64 &kl) {
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
// The reference's relaxed keys keep, of the CSs that share a key in a level, the one its
// threads insert first: blocks run in order and, within a block, roughly thread order (the
// oracle's sequential tid order).  Here the row of a key records the priority (block position
// << 40 | the reference's thread index, U's "l U r" before "r U l") of the candidate it holds;
// a candidate of the same level with the same key and a lower priority takes the row over: it
// locks the priority word (bit 0), rewrites the row and its parent, and publishes its
// priority.  Rows of lower levels are never taken over.  So a shared key never goes to a later
// block, which keeps the per-block stored counts equal to the oracle's; inside a block the
// thread index counts operand rows in the order they were stored, which on the device (as in
// the reference) is the order warps reached the hash set.  One lane, bounded waits.
template <class Gen>
__device__ void take_over(const InstArgs &A, InstCtl *C, const Gen &g, int t, u64 row, u64 prio, u64 parent) {
    u64 *pw = A.prio + row;
    const int nch = A.pitch >> 1;
    for (long long spin = 0; spin < A.wait_spins; ++spin) {
        const u64 v = ld_acquire(pw);
        if ((v >> 1) <= prio) return;  // the row holds an earlier candidate (or this one)
        if (v & 1ull) {                // another take-over is writing the row
            __nanosleep(128);
            continue;
        }
        if (atomicCAS(pw, v, (prio << 1) | 1ull) != v) continue;
        ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(A.cache + row * (u64)A.pitch);
        for (int c = 0; c < nch; ++c) dst[c] = g.word(t, c, g.pre(c));
        A.parents[row] = parent;
        __threadfence();
        st_release(pw, prio << 1);
        return;
    }
    atomicOr(&C->status, ST_WAIT);
}

template <int NC, class Gen>
__device__ __forceinline__ void resolve(const InstArgs &A, InstCtl *C, int cost, const Gen &g, u64 fp, bool active,
                                        u64 parent, u64 kh, u64 kl, u64 prio, u32 anyp, u32 anyn, int *overflowed,
                                        int lane) {
    int state = active ? S_PROBE : S_DONE;
    const u64 tagbits = (fp >> 40) << 40;
    const u64 genbits = (u64)A.gen << 32;
    const u64 want = tagbits | genbits | FIELD_PENDING;
    const u64 mask = A.slot_mask;
    u64 idx = fp & mask;
    long long vrow = -1;
    u64 probes = 0;
    const int nch = A.pitch >> 1;
    const u64 pitch = (u64)A.pitch;
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
                    if (A.key_mode == KEY_EXACT) prefetch_l2(A.cache + (u64)vrow * pitch, (u32)(pitch * 8));
                    state = S_VERIFY;
                    break;
                }
                idx = (idx + 1) & mask;
                if (++probes > mask) {
                    atomicOr(&C->status, ST_TABLE);
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
            if (lane == leader) base = atomicAdd(&C->row_count, (u64)__popc(cm));
            base = __shfl_sync(FULL, base, leader);
            const u64 cap = (u64)A.cap_rows;
            // WU chunks per lane are loaded before any of their words is stored: the stores go
            // to the same cache as the loads, so the compiler keeps them in program order
            for (int c0 = lane; c0 < nch; c0 += 32 * WU) {
                typename Gen::Pre pv[WU];
#pragma unroll
                for (int u = 0; u < WU; ++u)
                    if (c0 + 32 * u < nch) pv[u] = g.pre(c0 + 32 * u);
#pragma unroll
                for (int u = 0; u < WU; ++u) {
                    const int c = c0 + 32 * u;
                    if (c >= nch) break;
#pragma unroll
                    for (int t = 0; t < NC; ++t) {
                        if ((cm >> t) & 1u) {
                            const u64 row = base + __popc(cm & ((1u << t) - 1u));
                            if (row < cap) reinterpret_cast<ulonglong2 *>(A.cache + row * pitch)[c] = g.word(t, c, pv[u]);
                        }
                    }
                }
            }
            const u64 myrow = base + __popc(cm & ((1u << lane) - 1u));
            if (A.lstats) count_row_stats(A.lstats + (u64)cost * LSTATS, state == S_CLAIM && myrow < cap, anyp, anyn, lane);
            if (state == S_CLAIM && myrow < cap) {
                A.parents[myrow] = parent;
                if (A.keys) {
                    A.keys[2 * myrow] = kh;
                    A.keys[2 * myrow + 1] = kl;
                }
                if (A.prio) A.prio[myrow] = prio << 1;
            }
            __threadfence();
            __syncwarp();
            if (state == S_CLAIM) {
                u32 f = FIELD_OVERFLOW;
                if (myrow < cap)
                    f = (u32)(myrow + 1);
                else if ((atomicOr(&C->status, ST_OVERFLOW) & ST_OVERFLOW) == 0u)
                    atomicCAS(&C->overflow_cost, 0u, (u32)cost);
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
                atomicOr(&C->status, ST_WAIT);
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
                u32 diff = 0;
                const u32 myv = (u32)vrow;
                const ulonglong2 *vr[NC];
#pragma unroll
                for (int t = 0; t < NC; ++t)
                    vr[t] = reinterpret_cast<const ulonglong2 *>(A.cache + (u64)__shfl_sync(FULL, myv, t) * pitch);
#pragma unroll 1
                for (int c = lane; c < nch; c += 32) {
                    const auto p = g.pre(c);
#pragma unroll
                    for (int t = 0; t < NC; ++t) {
                        if ((vm >> t) & 1u) {
                            const ulonglong2 a = g.word(t, c, p);
                            const ulonglong2 b = __ldcg(vr[t] + c);
                            diff |= (u32)((a.x != b.x) | (a.y != b.y)) << t;
                        }
                    }
                }
                const u32 anydiff = __reduce_or_sync(FULL, diff);
                if (state == S_VERIFY) {
                    if ((anydiff >> lane) & 1u) {
                        state = S_PROBE;
                        idx = (idx + 1) & mask;
                    } else {
                        state = S_DONE;
                    }
                }
            }
        } else if (state == S_VERIFY) {
            const u64 eh = __ldcg(A.keys + 2 * vrow), el = __ldcg(A.keys + 2 * vrow + 1);
            if (eh == kh && el == kl) {
                if (A.prio && vrow >= __ldcg(A.ls + cost)) take_over(A, C, g, lane, (u64)vrow, prio, parent);
                state = S_DONE;
            } else {
                state = S_PROBE;
                idx = (idx + 1) & mask;
            }
        }
    }
}

// Fingerprints, acceptance, the find record, uniqueness for NC candidates of one warp.
// pos_of(t): block position of candidate t (the find record is per block).
template <int NC, class Gen, class ParentOf, class PosOf, class TidOf>
__device__ __forceinline__ void finish(const InstArgs &A, InstCtl *C, Slot &sl, const Gen &g, u64 (&h)[NC], u32 bp,
                                       u32 bn, u32 valid, ParentOf parent_of, PosOf pos_of, TidOf tid_of, int lane) {
    const u64 sum = reduce_to_lane<NC>(h, lane);
    const u32 anyp = __reduce_or_sync(FULL, bp), anyn = __reduce_or_sync(FULL, bn);
    const u32 acc = ~(anyp | anyn) & valid;
    const u64 myparent = parent_of(lane);
    const int cost = sl.cost;
    if (acc) {
        if ((acc >> lane) & 1u) {
            const int p = pos_of(lane);
            const u64 key = ((u64)cost << 32) | (u32)p;
            if (key < ld_volatile(&C->found_key)) {  // else a block at or before this one holds a find
                atomicCAS(A.found_par + p, 0ull, (1ull << 63) | myparent);
                atomicMin(&C->found_key, key);
            }
            // the item's remaining rows are skipped only when the search ends at this level
            if (A.stop_at_found && (A.find_first || sl.pos >= p)) sl.stop = 1;
        }
        __syncwarp();
        if (A.stop_at_found) return;  // this level is the last one; its candidates need no dedupe
    }
    if (sl.check_only) return;
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
    const u64 prio = A.prio && ((valid >> lane) & 1u) ? ((u64)(u32)pos_of(lane) << 40) | tid_of(lane) : 0ull;
    // once the language cache has overflowed, the level's remaining CSs are not stored and take
    // no hash slots
    const bool room = *(volatile int *)&sl.overflowed == 0;
    resolve<NC>(A, C, cost, g, fp, room && ((valid >> lane) & 1u), myparent, kh, kl, prio, anyp, anyn, &sl.overflowed,
                lane);
}

// ---------------------------------------------------------------- rows
// Binary row: right row r (at R) against the slot's tile of TLP left rows (U: both orders of
// each pair, TL = 2 TLP candidates; & and |: TL = TLP).  Chunks are 16 bytes (two words); two
// are in flight per lane.  Positives are the first npos words, so acceptance needs no metadata.
template <int OPC, int TL, int HK>
__device__ __forceinline__ void binary_row(const InstArgs &A, InstCtl *C, Slot &sl, const ulonglong2 *tile,
                                           int nl, long long l_first, const ulonglong2 *R, long long r, int lane) {
    constexpr int TLP = OPC == OP_U ? TL / 2 : TL;
    constexpr int NC = TL;
    const int nch = A.pitch >> 1, npos = A.npos, n = A.n;
    const int rop = sl.op;
    u64 h[NC];
#pragma unroll
    for (int t = 0; t < NC; ++t) h[t] = 0;
    u32 bp = 0, bn = 0;
    constexpr int CH = 2;  // right-row chunks in flight per lane
    for (int c0 = lane; c0 < nch; c0 += 32 * CH) {
        ulonglong2 rvv[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int c = c0 + 32 * u;
            if (c < nch) rvv[u] = __ldcg(R + c);
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int c = c0 + 32 * u;
            if (c >= nch) continue;
            const u64 k = (2ull * (u64)c + 1ull) * WEYL;
            const ulonglong2 rv = rvv[u];
            const u64 p0 = 2 * c < npos ? 1ull : 0ull, p1 = 2 * c + 1 < npos ? 1ull : 0ull;
            const bool v0 = 2 * c < n, v1 = 2 * c + 1 < n;
            const u64 rx = OPC == OP_U ? rev62(rv.x) : 0ull, ry = OPC == OP_U ? rev62(rv.y) : 0ull;
#pragma unroll
            for (int t = 0; t < TLP; ++t) {
                if (t < nl) {
                    const ulonglong2 lv = tile[t * nch + c];
                    if (OPC == OP_U) {
                        const u64 lx = rev62(lv.x), ly = rev62(lv.y);
                        const u64 ax = lx | rx, ay = ly | ry;
                        const u64 a0 = until_rev(ax, rx), a1 = until_rev(ay, ry);  // l U r
                        const u64 b0 = until_rev(ax, lx), b1 = until_rev(ay, ly);  // r U l
                        h[2 * t] += hw<HK>(a0, k, v0) + hw<HK>(a1, k + WEYL, v1);
                        h[2 * t + 1] += hw<HK>(b0, k, v0) + hw<HK>(b1, k + WEYL, v1);
                        bp |= (pmiss2(a0, a1, p0, p1) << (2 * t)) | (pmiss2(b0, b1, p0, p1) << (2 * t + 1));
                        bn |= (nhit2(a0, a1, p0, p1) << (2 * t)) | (nhit2(b0, b1, p0, p1) << (2 * t + 1));
                    } else {
                        const u64 w0 = rop == OP_AND ? (lv.x & rv.x) : (lv.x | rv.x);
                        const u64 w1 = rop == OP_AND ? (lv.y & rv.y) : (lv.y | rv.y);
                        h[t] += hw<HK>(w0, k, v0) + hw<HK>(w1, k + WEYL, v1);
                        bp |= pmiss2(w0, w1, p0, p1) << t;
                        bn |= nhit2(w0, w1, p0, p1) << t;
                    }
                }
            }
        }
    }
    const int cnt = OPC == OP_U ? 2 * nl : nl;
    const u32 valid = cnt >= 32 ? FULL : ((1u << cnt) - 1u);
    const BinGen<OPC> g{tile, R, nch, rop};
    finish<NC>(A, C, sl, g, h, bp, bn, valid,
               [&](int t) {
                   if (OPC == OP_U) {
                       const u64 l = (u64)(l_first + (t >> 1));
                       return (t & 1) ? pack_parent(OP_U, (u64)r, l) : pack_parent(OP_U, l, (u64)r);
                   }
                   return pack_parent(rop, (u64)(l_first + t), (u64)r);
               },
               [&](int) { return sl.pos; },
               [&](int t) -> u64 {  // the reference's thread index: (l - l0) * R + (r - r0); U: both orders
                   const u64 l = (u64)(l_first + (OPC == OP_U ? (t >> 1) : t));
                   const u64 tid = (l - (u64)sl.e_l0) * (u64)sl.e_R + ((u64)r - (u64)sl.e_r0);
                   return OPC == OP_U ? 2 * tid + (u64)(t & 1) : tid;
               },
               lane);
    if (lane == 0) atomicAdd(&sl.evals, (unsigned)cnt);
}

// Unary row: every operator of the slot's mask on source row s (at src; one load of each chunk).
template <int HK>
__device__ __forceinline__ void unary_row(const InstArgs &A, InstCtl *C, Slot &sl, int mask, const ulonglong2 *src,
                                          long long s, int lane) {
    constexpr int NC = 4;
    const int nch = A.pitch >> 1, npos = A.npos, n = A.n;
    const ulonglong2 *meta = reinterpret_cast<const ulonglong2 *>(A.wmeta);
    u64 h[NC] = {0, 0, 0, 0};
    u32 bp = 0, bn = 0;
    constexpr int CH = 2;  // source-row chunks in flight per lane
    for (int c0 = lane; c0 < nch; c0 += 32 * CH) {
        ulonglong2 sv[CH], mv[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int c = c0 + 32 * u;
            if (c < nch) {
                sv[u] = __ldcg(src + c);
                mv[u] = __ldcg(meta + c);  // a batch slot rewrites its metadata in the launch
            }
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int c = c0 + 32 * u;
            if (c >= nch) continue;
            const u64 k = (2ull * (u64)c + 1ull) * WEYL;
            const u64 p0 = 2 * c < npos ? 1ull : 0ull, p1 = 2 * c + 1 < npos ? 1ull : 0ull;
            const bool v0 = 2 * c < n, v1 = 2 * c + 1 < n;
            const u64 m0 = mv[u].x & LENMASK, m1 = mv[u].y & LENMASK;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if ((mask >> j) & 1) {
                    const int op = unary_slot_op(j);
                    const u64 w0 = unary_word(op, sv[u].x, m0), w1 = unary_word(op, sv[u].y, m1);
                    h[j] += hw<HK>(w0, k, v0) + hw<HK>(w1, k + WEYL, v1);
                    bp |= pmiss2(w0, w1, p0, p1) << j;
                    bn |= nhit2(w0, w1, p0, p1) << j;
                }
            }
        }
    }
    const u32 valid = (u32)(mask & 15);
    const UnGen g{src, meta};
    finish<NC>(A, C, sl, g, h, bp, bn, valid,
               [&](int t) { return pack_parent(unary_slot_op(t & 3), (u64)s, 0); },
               [&](int t) { return sl.upos[t & 3]; }, [&](int) -> u64 { return (u64)(s - sl.e_r0); }, lane);
    if (lane == 0) atomicAdd(&sl.evals, (unsigned)__popc(valid));
}

// ---------------------------------------------------------------- planner (one warp)
__device__ __forceinline__ long long ls_at(const InstArgs &A, int k) { return __ldcg(A.ls + k); }

// Rows of cost k < c: [lo, hi); empty outside c1 .. c - 1.
__device__ __forceinline__ void level_range(const InstArgs &A, int k, int c, long long &lo, long long &hi) {
    if (k < A.cf[0] || k >= c) {
        lo = hi = 0;
        return;
    }
    lo = ls_at(A, k);
    hi = ls_at(A, k + 1);
}

__device__ __forceinline__ void store_entry(Entry *dst, const Entry &e) {
    const u64 *s = reinterpret_cast<const u64 *>(&e);
    u64 *d = reinterpret_cast<u64 *>(dst);
#pragma unroll
    for (int w = 0; w < (int)(sizeof(Entry) / 8); ++w) __stcg(d + w, s[w]);
}

// The binary blocks of operator op (cost cop) of level c, in the reference's split order
// (i = c1 .. (c - cop) / 2 over non-empty levels i and j = c - i - cop): written as entries
// from queue index *eidx and positions from *pos.  Returns the candidates of this lane's blocks.
__device__ u64 plan_binary(const InstArgs &A, int c, int op, int ne_count, int ne_lane, int &pos, int &eidx,
                           u64 &units, int lane) {
    const int cop = A.cf[op + 1], c1 = A.cf[0];
    const int tl = op == OP_U ? max(1, A.tile / 2) : A.tile;
    u64 cand = 0;
    if (c - cop < 2 * c1) return 0;
    for (int base = 0; base < ne_count; base += 32) {
        const int q = base + lane;
        const int i = q < ne_count ? (base == 0 ? ne_lane : __ldcg(A.ne + q)) : 0;
        const bool ok_i = q < ne_count && i >= c1 && 2 * i <= c - cop;
        long long li = 0, hi_ = 0, lj = 0, hj = 0;
        if (ok_i) {
            level_range(A, i, c, li, hi_);
            level_range(A, c - i - cop, c, lj, hj);
        }
        const bool ex = ok_i && hi_ > li && hj > lj;
        const u32 m = __ballot_sync(FULL, ex);
        if (ex) {
            const int rank = __popc(m & ((1u << lane) - 1u));
            Entry e{};
            e.kind = op == OP_U ? ENT_U : ENT_ANDOR;
            e.op = op;
            e.pos = pos + rank;
            for (int j = 0; j < 4; ++j) e.upos[j] = POS_NONE;
            e.lcost = i;
            e.rcost = c - i - cop;
            e.l0 = li;
            e.l1 = hi_;
            e.r0 = lj;
            e.r1 = hj;
            e.cand = (u64)(op == OP_U ? 2 : 1) * (u64)(hi_ - li) * (u64)(hj - lj);
            cand += e.cand;
            units += (u64)((hi_ - li + tl - 1) / tl) * (u64)(hj - lj);
            store_entry(A.entries + eidx + rank, e);
        }
        pos += __popc(m);
        eidx += __popc(m);
        if (__any_sync(FULL, q < ne_count && 2 * i > c - cop)) break;  // the list is sorted by cost
    }
    return cand;
}

// Builds the plan of level c in the reference's block order (ltli6463.cu:1209-1440): ~, &
// splits, | splits, X, F, G, U splits (NegType rule :1212).  The queue runs the unary entries
// first (fused over operators that read the same source rows), then the & / | / U blocks.
// One warp; writes the entries and C->plan (not yet published).
__device__ void plan_level(const InstArgs &A, InstCtl *C, int c, int lane) {
    const int c1 = A.cf[0];
    const int ne_count = (int)__ldcg(&C->ne_count);
    const u64 found_key = __ldcg(&C->found_key);  // loaded early: nothing changes it while planning
    // the first 32 non-empty levels, one per lane, for all three binary operators
    const int ne_lane = lane < ne_count ? __ldcg(A.ne + lane) : 0;
    // unary operators: lane j < 4 looks at slot operator j
    bool uex = false;
    long long ulo = 0, uhi = 0;
    int uk = 0;
    if (lane < 4) {
        const int op = unary_slot_op(lane);
        uk = c - A.cf[op + 1];
        bool ok = uk >= c1;
        if (op == OP_NEG) ok = (A.neg_type == 1 && uk >= c1) || (A.neg_type == 2 && uk == c1);
        if (ok) level_range(A, uk, c, ulo, uhi);
        uex = ok && uhi > ulo;
    }
    const u32 um = __ballot_sync(FULL, uex) & 15u;
    long long lo4[4], hi4[4];
    int k4[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        lo4[j] = __shfl_sync(FULL, ulo, j);
        hi4[j] = __shfl_sync(FULL, uhi, j);
        k4[j] = __shfl_sync(FULL, uk, j);
    }
    // unary entries: one per distinct source range (fused) or per operator
    const bool fuse = !(A.plan_flags & PLAN_UNFUSED);
    int group[4], nu = 0;
    for (int j = 0; j < 4; ++j) {
        group[j] = -1;
        if (!((um >> j) & 1u)) continue;
        for (int q = 0; q < j && fuse; ++q)
            if (group[q] >= 0 && lo4[q] == lo4[j] && hi4[q] == hi4[j]) group[j] = group[q];
        if (group[j] < 0) group[j] = nu++;
    }
    // positions in the reference's order, binary entries after the unary ones in the queue
    int pos = 0, eidx = nu;
    int upos[4] = {POS_NONE, POS_NONE, POS_NONE, POS_NONE};
    if (um & 1u) upos[0] = pos++;
    u64 units_b = 0, units_u = 0;  // binary: (left tile, right row) pairs; unary: source rows
    u64 cand = plan_binary(A, c, OP_AND, ne_count, ne_lane, pos, eidx, units_b, lane);
    cand += plan_binary(A, c, OP_OR, ne_count, ne_lane, pos, eidx, units_b, lane);
    for (int j = 1; j < 4; ++j)
        if ((um >> j) & 1u) upos[j] = pos++;
    cand += plan_binary(A, c, OP_U, ne_count, ne_lane, pos, eidx, units_b, lane);
    if (lane == 0) {
        for (int g = 0; g < nu; ++g) {
            Entry e{};
            e.kind = ENT_UNARY;
            e.pos = POS_NONE;
            for (int j = 0; j < 4; ++j) {
                e.upos[j] = POS_NONE;
                if (group[j] != g) continue;
                e.opmask |= 1 << j;
                e.upos[j] = upos[j];
                e.pos = min(e.pos, upos[j]);
                e.lcost = k4[j];
                e.r0 = lo4[j];
                e.r1 = hi4[j];
                e.cand += (u64)(hi4[j] - lo4[j]);
            }
            cand += e.cand;
            units_u += (u64)(e.r1 - e.r0);
            store_entry(A.entries + g, e);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cand += __shfl_xor_sync(FULL, cand, o);
        units_b += __shfl_xor_sync(FULL, units_b, o);
        units_u += __shfl_xor_sync(FULL, units_u, o);
    }
    const int nent = eidx, nblocks = pos;
    __threadfence_block();
    // Item sizes: a level with fewer candidates than small_level is cut into items of about
    // units / item_target rows (at least small_rows), so every SM's slots take part and each
    // claim brings a few rows; larger levels use the big sizes.
    const bool small = (long long)cand < A.small_level;
    const long long tgt = max(1ll, A.item_target);
    const int rc = small ? (int)max((long long)max(1, A.small_rows),
                                    min((long long)A.right_chunk_big, ((long long)units_b + tgt - 1) / tgt))
                         : max(1, A.right_chunk_big);
    const int ur = small ? (int)max((long long)max(1, A.small_rows),
                                    min((long long)A.unary_rows_big, ((long long)units_u + tgt - 1) / tgt))
                         : max(1, A.unary_rows_big);
    long long items = 0;
    for (int base = 0; base < nent; base += 32) {
        const int e = base + lane;
        long long it = 0, tiles_r = 1;
        Entry *pe = A.entries + e;
        if (e < nent) {
            const int kind = __ldcg(&pe->kind);
            const long long l0 = __ldcg(&pe->l0), l1 = __ldcg(&pe->l1), r0 = __ldcg(&pe->r0), r1 = __ldcg(&pe->r1);
            if (kind == ENT_UNARY) {
                it = (r1 - r0 + ur - 1) / ur;
            } else {
                const int tl = kind == ENT_U ? max(1, A.tile / 2) : A.tile;
                tiles_r = (r1 - r0 + rc - 1) / rc;
                it = ((l1 - l0 + tl - 1) / tl) * tiles_r;
            }
        }
        // exclusive prefix of the item counts over the warp
        long long incl = it;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        if (e < nent) {
            __stcg(&pe->item0, items + incl - it);
            __stcg(&pe->items, it);
            __stcg(&pe->tiles_r, tiles_r);
        }
        items += __shfl_sync(FULL, incl, 31);
    }
    // the find record of the level's blocks starts empty (unless an earlier level holds the find)
    if (found_key == NO_FIND)
        for (int p = lane; p < nblocks; p += 32) __stcg(A.found_par + p, 0ull);
    if (lane == 0) {
        Plan &P = C->plan;
        P.cost = c;
        P.halt = 0;
        P.check_only = A.on_the_fly;
        P.nentries = nent;
        P.nblocks = nblocks;
        P.right_chunk = rc;
        P.unary_rows = ur;
        P.learned = 0;
        P.items = items;
        P.cand = cand;
        A.level_cands[c] = cand;
    }
    __syncwarp();
}

// Learned order (PLAN_LEARNED): every block of the plan is scored by the scorer, one block
// at a time on this warp (lane l computes hidden units l and l + 32).  A fused unary entry's
// chance is that any of its operators' blocks accepts, 1 - prod(1 - p).  Entries are sorted by
// chance / sqrt(candidates), highest first, ties in the reference's order, and their item
// starts are laid out again in the new order.  Plans whose items all start at once
// (learn_min_items) keep the plain order.
__device__ void score_plan(const InstArgs &A, InstCtl *C, int lane) {
    const int ne = __ldcg(&C->plan.nentries);
    if (ne <= 1 || __ldcg(&C->plan.items) <= A.learn_min_items || !A.model) return;
    const MlpDev &M = *reinterpret_cast<const MlpDev *>(A.model);
    const int c = __ldcg(&C->plan.cost), nblocks = __ldcg(&C->plan.nblocks);
    const long long level_cands = (long long)__ldcg(&C->plan.cand);
    for (int e = 0; e < ne; ++e) {
        const Entry *E = A.entries + e;
        const int kind = __ldcg(&E->kind), opmask = __ldcg(&E->opmask), lcost = __ldcg(&E->lcost);
        const long long l0 = __ldcg(&E->l0), l1 = __ldcg(&E->l1), r0 = __ldcg(&E->r0), r1 = __ldcg(&E->r1);
        const long long cand = (long long)__ldcg(&E->cand);
        float miss = 1.0f;
        for (int j = 0; j < 4; ++j) {
            int op, position;
            long long lrows, rrows, bc;
            if (kind == ENT_UNARY) {
                if (!((opmask >> j) & 1)) continue;
                op = unary_slot_op(j);
                position = __ldcg(&E->upos[j]);
                lrows = r1 - r0;
                rrows = 1;
                bc = r1 - r0;
            } else {
                if (j) break;
                op = __ldcg(&E->op);
                position = __ldcg(&E->pos);
                lrows = l1 - l0;
                rrows = r1 - r0;
                bc = cand;
            }
            const BlockInfo bi = block_info(op, c, lcost, lrows, rrows, bc, position, A.cf, nblocks, level_cands,
                                            A.lstats, A.max_cost, A.npos, A.n, A.nalpha);
            float f[ORDER_NF];
            block_features(bi, f);
            const float z = mlp_score_warp(M, f, lane);
            miss *= 1.0f / (1.0f + expf(z));  // 1 - sigmoid(z)
        }
        if (lane == 0) __stcg(&A.entries[e].score, (1.0f - miss) / sqrtf((float)(cand > 0 ? cand : 1)));
    }
    __syncwarp();
    __threadfence_block();
    Entry *scratch = A.entries + A.cap_entries;
    for (int e = lane; e < ne; e += 32) {
        const float ke = __ldcg(&A.entries[e].score);
        const int pe = __ldcg(&A.entries[e].pos);
        int r = 0;
        for (int j = 0; j < ne; ++j) {
            const float kj = __ldcg(&A.entries[j].score);
            r += (kj > ke || (kj == ke && __ldcg(&A.entries[j].pos) < pe)) ? 1 : 0;
        }
        Entry x;
        constexpr int W = sizeof(Entry) / 8;
        for (int w = 0; w < W; ++w) reinterpret_cast<u64 *>(&x)[w] = __ldcg(reinterpret_cast<const u64 *>(A.entries + e) + w);
        store_entry(scratch + r, x);
    }
    __syncwarp();
    __threadfence_block();
    long long item0 = 0;
    for (int base = 0; base < ne; base += 32) {
        const int e = base + lane;
        Entry x{};
        long long it = 0;
        if (e < ne) {
            constexpr int W = sizeof(Entry) / 8;
            for (int w = 0; w < W; ++w) reinterpret_cast<u64 *>(&x)[w] = __ldcg(reinterpret_cast<const u64 *>(scratch + e) + w);
            it = x.items;
        }
        long long incl = it;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        if (e < ne) {
            x.item0 = item0 + incl - it;
            store_entry(A.entries + e, x);
        }
        item0 += __shfl_sync(FULL, incl, 31);
    }
    if (lane == 0) C->plan.learned = 1;
    __syncwarp();
}

// Publishes the plan in C->plan: counters reset, then the claim limit and the claim counter
// with the new sequence number (release).  A plan that is not opened hands out no item until
// the host sets the limit (host-driven levels: the host may reorder the plan or run it in
// windows first).  Lane 0.
__device__ __forceinline__ void publish(InstCtl *C, long long items, bool open) {
    const u32 seq = __ldcg(&C->seq) + 1;
    __threadfence();  // the plan and entries (written by the whole warp) come first
    C->done = 0;
    C->limit = ((u64)seq << SEQ_SHIFT) | (u64)(open ? items : 0);
    st_release(&C->claimed, (u64)seq << SEQ_SHIFT);  // orders done and limit before the new sequence
    st_release32(&C->seq, seq);
}

// Closes the current level (its last item is done) and plans the next level with items,
// stopping when the search is over.  Levels without any block are closed on the spot.  One
// warp (all lanes).  With open false (host-driven levels) the next plan is made but hands out
// nothing until the host opens it.
__device__ bool close_level(const InstArgs &A, InstCtl *C, bool open, int lane) {
    __threadfence();
    int c = (int)__ldcg(&C->plan.cost);
    bool halt = false;
    for (;;) {
        if (lane == 0) {
            const long long rows = min((long long)__ldcg(&C->row_count), A.cap_rows);
            A.ls[c + 1] = rows;
            if (rows > __ldcg(A.ls + c)) {
                const u32 k = __ldcg(&C->ne_count);
                A.ne[k] = c;
                C->ne_count = k + 1;
            }
            if (A.level_ns) A.level_ns[(u64)c * LEVEL_TRACE + LT_END] = globaltimer();
            C->last_cost = (u32)c;
            const u64 fk = __ldcg(&C->found_key);
            if (fk != NO_FIND && (int)(fk >> 32) == c && __ldcg(&C->found) == 0ull) {
                C->found = __ldcg(A.found_par + (u32)fk);
                C->found_cost = (u32)c;
            }
        }
        __syncwarp();
        __threadfence();
        const u32 st = __ldcg(&C->status);
        const u32 bad = ST_FATAL | (A.on_the_fly ? 0u : ST_OVERFLOW);
        const bool cancelled = A.cancel && *A.cancel != 0u;
        halt = c + 1 > A.max_cost || (A.stop_at_found && __ldcg(&C->found) != 0ull) || (st & bad) != 0u || cancelled;
        if (halt) {
            if (lane == 0) {
                C->plan.halt = 1;
                C->plan.items = 0;
                atomicOr(&C->flags, CTL_DONE | (cancelled ? CTL_CANCELLED : 0u));
                publish(C, 0, false);
            }
            __syncwarp();
            return true;
        }
        ++c;
        plan_level(A, C, c, lane);
        if (A.plan_flags & PLAN_LEARNED) score_plan(A, C, lane);
        const long long items = __ldcg(&C->plan.items);
        if (items > 0) {
            if (lane == 0) {
                publish(C, items, open);
                if (A.level_ns) A.level_ns[(u64)c * LEVEL_TRACE + LT_PUBLISHED] = globaltimer();
            }
            __syncwarp();
            return false;
        }
        // a level without blocks: it ends where it starts
    }
}

// ---------------------------------------------------------------- batches
// Candidates the reference counts in level c up to and including the block at position fpos of
// its block order (ltli6463.cu:1209-1440; only blocks whose operand levels are non-empty have
// positions).  Lane 0.
__device__ u64 count_blocks_through(const InstArgs &A, int c, int fpos) {
    const int c1 = A.cf[0];
    u64 all = 0;
    int pos = 0;
    auto size = [&](int k) -> long long { return (k >= c1 && k < c) ? ls_at(A, k + 1) - ls_at(A, k) : 0ll; };
    auto take = [&](long long n) {
        if (n <= 0 || pos > fpos) return;
        all += (u64)n;
        ++pos;
    };
    auto binary = [&](int cop, long long mult) {
        for (int i = c1; 2 * i <= c - cop; ++i) {
            const long long a = size(i), b = size(c - i - cop);
            if (a > 0 && b > 0) take(mult * a * b);
        }
    };
    const int *cf = A.cf;
    if ((A.neg_type == 1 && c - cf[1] >= c1) || (A.neg_type == 2 && c - cf[1] == c1)) take(size(c - cf[1]));
    binary(cf[2], 1);
    binary(cf[3], 1);
    if (c - cf[4] >= c1) take(size(c - cf[4]));
    if (c - cf[5] >= c1) take(size(c - cf[5]));
    if (c - cf[6] >= c1) take(size(c - cf[6]));
    binary(cf[7], 2);
    return all;
}

__device__ __forceinline__ void load_args(InstArgs &A, const InstArgs *src) {
    constexpr int AW = sizeof(InstArgs) / 8;
    for (int w = 0; w < AW; ++w) reinterpret_cast<u64 *>(&A)[w] = __ldcg(reinterpret_cast<const u64 *>(src) + w);
}

// The result of slot s's instance, as ltlg_engine_learn reports it: status, cost, the
// reference's candidate count, and the found candidate's tree (row, parents) breadth first.
// One warp; lane 0 writes.
__device__ void finish_instance(BatchDev &B, int s, int lane) {
    if (lane == 0) {
        InstArgs A;
        load_args(A, B.args + s);
        InstCtl *C = A.ctl;
        const int idx = B.cur[s];
        BatchOut &o = B.out[idx];
        const int c1 = A.cf[0];
        const u32 st = __ldcg(&C->status), flags = __ldcg(&C->flags);
        const u64 found = __ldcg(&C->found);
        const int found_cost = (int)__ldcg(&C->found_cost);
        const int last_cost = max(c1, (int)__ldcg(&C->last_cost));
        const int letter = __ldcg(&o.letter);
        int status = LTLG_NOT_FOUND;
        if (st & ST_FATAL)
            status = (st & ST_TABLE) ? LTLG_TABLE_FULL : LTLG_DEVICE_WAIT;
        else if (found || letter >= 0)
            status = LTLG_FOUND;
        else if (flags & CTL_CANCELLED)
            status = LTLG_TIMEOUT;
        else if (st & ST_OVERFLOW)
            status = LTLG_NO_MEMORY;  // the slot's cache overflowed: the host learns it alone
        const bool stop_found = found && A.stop_at_found;
        const int top = stop_found ? found_cost : last_cost;
        u64 all = (u64)A.nalpha;
        for (int c = c1 + 1; c <= top; ++c)
            if (!(stop_found && c == found_cost)) all += __ldcg(A.level_cands + c);
        if (stop_found) all += count_blocks_through(A, found_cost, (int)(u32)__ldcg(&C->found_key));
        o.status = status;
        o.cost = letter >= 0 ? c1 : found ? found_cost : last_cost;
        o.all_ltls = all;
        o.evaluated = (u64)A.nalpha + __ldcg(&C->evaluated);
        o.rows = min((long long)__ldcg(&C->row_count), A.cap_rows);
        o.found = letter >= 0 ? 0ull : found;
        o.device_flags = st;
        o.ns = globaltimer() - B.t0[s];
        // the tree of the find, breadth first (entry 0 is the root)
        int count = 0, overflow = 0;
        if (found && letter < 0) {
            u64 *e = o.walk;
            e[0] = ~0ull;
            e[1] = found & ~(1ull << 63);
            count = 1;
            for (int head = 0; head < count && !overflow; ++head) {
                const u64 p = e[2 * head + 1];
                const int op = parent_op(p);
                const u64 kids[2] = {parent_left(p), parent_right(p)};
                const int nk = (op == OP_AND || op == OP_OR || op == OP_U) ? 2 : (op == OP_ATOM ? 0 : 1);
                for (int q = 0; q < nk; ++q) {
                    if (kids[q] < (u64)A.nalpha) continue;
                    if (count >= WALK_MAX) {
                        overflow = 1;
                        break;
                    }
                    e[2 * count] = kids[q];
                    e[2 * count + 1] = __ldcg(A.parents + kids[q]);
                    ++count;
                }
            }
        }
        o.walk_count = count;
        o.walk_overflow = overflow;
        __threadfence();
    }
    __syncwarp();
}

// Sets slot s up with instance idx: letters (the first separating one may end the search here,
// ltli6463.cu:1100-1136), word metadata, the slot's next hash-set generation, a clean control
// block and level arrays, the letters in the hash set, then the first plan.  One warp.  Returns
// true when the instance's levels run; false when its search ended at set-up (result written).
template <int HK>
__device__ bool setup_instance(BatchDev &B, int s, int idx, int lane) {
    BatchIn in;
    {
        const u64 *src = reinterpret_cast<const u64 *>(B.in + idx);
        for (int w = 0; w < (int)(sizeof(BatchIn) / 8); ++w) reinterpret_cast<u64 *>(&in)[w] = __ldcg(src + w);
    }
    InstArgs A;
    load_args(A, B.args + s);
    InstCtl *C = A.ctl;
    BatchOut &o = B.out[idx];
    const int npos = in.npos, n = in.npos + in.nneg, nalpha = in.nalpha;
    const int pitch = n <= 4 ? 4 : ((n + 3) & ~3);
    const int c1 = A.cf[0];
    if (lane == 0) {
        B.cur[s] = idx;
        B.t0[s] = globaltimer();
        o.letter = -1;
        o.walk_count = 0;
        o.walk_overflow = 0;
        o.found = 0;
    }
    const u32 *steps = B.steps + in.steps0;
    const int *offs = B.offs + in.offs0;
    // letters: rows 0 .. nalpha - 1, positives need position 0, negatives must not hold there
    int hit = -1;
    u64 all = 0;
    for (int j = 0; j < nalpha; ++j) {
        const u32 bit = 1u << (in.alpha[j] - 'a');
        bool acc = true;
        for (int i = lane; i < pitch; i += 32) {
            u64 w = 0;
            if (i < n) {
                const int a = offs[i], b = offs[i + 1];
                for (int k = a; k < b; ++k)
                    if (steps[k] & bit) w |= 1ull << (k - a);
                if (i < npos ? !(w & 1ull) : (w & 1ull)) acc = false;
            }
            __stcg(A.cache + (u64)j * pitch + i, w);
        }
        acc = __all_sync(FULL, acc);
        ++all;
        if (acc && hit < 0) {
            hit = j;
            if (A.stop_at_found) break;
        }
    }
    if (hit >= 0 && lane == 0) o.letter = hit;
    if ((hit >= 0 && A.stop_at_found) || n == 0 || nalpha == 0) {
        if (lane == 0) {
            o.status = hit >= 0 ? LTLG_FOUND : LTLG_NOT_FOUND;
            o.cost = hit >= 0 ? c1 : max(c1, A.max_cost);
            o.all_ltls = all;
            o.evaluated = all;
            o.rows = hit >= 0 && A.stop_at_found ? hit + 1 : 0;  // no rows of an instance without traces
            o.device_flags = 0;
            o.ns = globaltimer() - B.t0[s];
            __threadfence();
        }
        __syncwarp();
        return false;
    }
    // word metadata: length mask | positive flag
    for (int i = lane; i < pitch; i += 32) {
        u64 m = 0;
        if (i < n) {
            const int ln = offs[i + 1] - offs[i];
            m = (ln >= 63 ? 0x7FFFFFFFFFFFFFFFull : ((1ull << ln) - 1)) | (i < npos ? (1ull << 63) : 0ull);
        }
        __stcg(const_cast<u64 *>(A.wmeta) + i, m);
    }
    // the slot's arguments for this instance; a generation that wraps clears the set
    A.n = n;
    A.pitch = pitch;
    A.npos = npos;
    A.nalpha = nalpha;
    A.rlx_type = 0;
    A.on_the_fly = 0;
    A.cap_rows = min(B.max_rows, B.cache_words / pitch);
    if (A.gen >= 255) {
        for (u64 q = lane; q <= A.slot_mask; q += 32) __stcg(A.slots + q, 0ull);
        A.gen = 1;
    } else {
        A.gen += 1;
    }
    {
        constexpr int AW = sizeof(InstArgs) / 8;
        for (int w = lane; w < AW; w += 32)
            __stcg(reinterpret_cast<u64 *>(B.args + s) + w, reinterpret_cast<const u64 *>(&A)[w]);
    }
    // level arrays and the control block (the plan sequence goes on: claim tags stay unique)
    for (int k = lane; k <= A.max_cost + 2; k += 32) {
        __stcg(A.ls + k, 0ll);
        __stcg(A.level_cands + k, 0ull);
    }
    if (lane == 0) {
        const u32 seq = __ldcg(&C->seq);
        C->claimed = (u64)seq << SEQ_SHIFT;
        C->limit = (u64)seq << SEQ_SHIFT;
        C->done = 0;
        C->row_count = (u64)nalpha;
        C->found_key = NO_FIND;
        C->found = 0;
        C->evaluated = 0;
        C->status = 0;
        C->found_cost = 0;
        C->overflow_cost = 0;
        C->ne_count = 0;
        C->last_cost = 0;
        C->flags = 0;
        C->t_start = globaltimer();
        C->plan.cost = c1;
        C->plan.halt = 0;
    }
    __threadfence();
    __syncwarp();
    // the letters into the hash set, in letter order (a duplicate letter stays a row, the set
    // keeps the first, as the reference's sequential inserts do: ltli6463.cu:1134, :1189-1190)
    const int nch = pitch >> 1;
    const u64 tagmask = ~((1ull << 40) - 1);
    for (int j = 0; j < nalpha; ++j) {
        const ulonglong2 *row = reinterpret_cast<const ulonglong2 *>(A.cache + (u64)j * pitch);
        u64 h[1] = {0};
        for (int c = lane; c < nch; c += 32) {
            const u64 k = (2ull * (u64)c + 1ull) * WEYL;
            const ulonglong2 w = __ldcg(row + c);
            h[0] += hw<HK>(w.x, k, 2 * c < n) + hw<HK>(w.y, k + WEYL, 2 * c + 1 < n);
        }
        const u64 fp = fmix64(reduce_to_lane<1>(h, lane));
        const u64 tagbits = fp & tagmask, genbits = (u64)A.gen << 32;
        u64 idx2 = fp & A.slot_mask;
        for (u64 probe = 0; probe <= A.slot_mask; ++probe, idx2 = (idx2 + 1) & A.slot_mask) {
            u64 v = 0;
            int action = 0;  // 0 next, 1 claimed, 2 compare
            if (lane == 0) {
                v = ld_acquire(A.slots + idx2);
                if (slot_free(v, A.gen)) {
                    const u64 old = atomicCAS(A.slots + idx2, v, tagbits | genbits | (u64)(j + 1));
                    if (old == v)
                        action = 1;
                    else
                        v = old;
                }
                if (action == 0 && (v & tagmask) == tagbits && (u32)v < FIELD_OVERFLOW) action = 2;
            }
            action = __shfl_sync(FULL, action, 0);
            v = __shfl_sync(FULL, v, 0);
            if (action == 1) break;
            if (action == 2) {
                const u64 other = (u64)(u32)v - 1;
                bool same;
                if (A.key_mode == KEY_EXACT) {
                    bool diff = false;
                    const ulonglong2 *ex = reinterpret_cast<const ulonglong2 *>(A.cache + other * pitch);
                    for (int c = lane; c < nch; c += 32) {
                        const ulonglong2 a = __ldcg(row + c), b = __ldcg(ex + c);
                        diff |= (a.x != b.x) | (a.y != b.y);
                    }
                    same = !__any_sync(FULL, diff);
                } else {
                    same = __ldcg(A.keys + 2 * other) == fp;
                }
                if (same) break;
            }
        }
        if (lane == 0) {
            A.parents[j] = pack_parent(OP_ATOM, 0, 0);
            if (A.keys) {
                A.keys[2 * j] = fp;
                A.keys[2 * j + 1] = 0;
            }
        }
        __threadfence();
        __syncwarp();
    }
    // the first plan: the letters' level has just ended
    const bool ended = close_level(A, C, true, lane);
    if (ended) finish_instance(B, s, lane);
    return !ended;
}

// Slot s takes pending instances until one has levels to run or none is left.  `live` counts the
// slots whose instance is searching: a slot that was searching (finishing) keeps its count when it
// takes another instance and drops it when none is left; a slot starting out adds it.  One warp.
template <int HK>
__device__ __noinline__ void next_instance(BatchDev &B, int s, bool finishing, int lane) {
    if (finishing) finish_instance(B, s, lane);
    for (;;) {
        u64 j = 0;
        if (lane == 0) j = atomicAdd(&B.next, 1ull);
        j = __shfl_sync(FULL, j, 0);
        if (j >= (u64)B.count) {
            if (finishing && lane == 0) atomicSub(&B.live, 1);
            __syncwarp();
            return;
        }
        if (setup_instance<HK>(B, s, (int)j, lane)) {
            if (!finishing && lane == 0) atomicAdd(&B.live, 1);
            __syncwarp();
            return;
        }
    }
}

// ---------------------------------------------------------------- the level kernel
__device__ __forceinline__ Slot *slot_at(unsigned char *smem, int s) { return reinterpret_cast<Slot *>(smem) + s; }

// Item `item` of entry e (cached in shared memory) into slot sl.  Returns the tile bytes to copy
// (0 for a unary item or a skipped one).
__device__ __forceinline__ u32 fill_slot(Slot &sl, int inst, const Entry &e, long long item, int tile, int rc,
                                         int ur, int cost, int check_only, long long plan_items, bool skip,
                                         int pitch) {
    const long long local = item - e.item0;
    sl.inst = inst;
    sl.kind = e.kind;
    sl.pos = e.pos;
    for (int j = 0; j < 4; ++j) sl.upos[j] = e.upos[j];
    sl.cost = cost;
    sl.check_only = check_only;
    sl.plan_items = plan_items;
    sl.next_row = 0;
    sl.rows_done = 0;
    sl.evals = 0;
    sl.stop = skip ? 1 : 0;
    sl.e_l0 = e.l0;
    sl.e_r0 = e.r0;
    sl.e_R = e.r1 - e.r0;
    if (e.kind == ENT_UNARY) {
        sl.op = e.opmask;
        sl.row0 = e.r0 + local * ur;
        sl.nrows = skip ? 1 : (int)min((long long)ur, e.r1 - sl.row0);
        sl.nl = 0;
        sl.l_first = 0;
        return 0;
    }
    const int tl = e.kind == ENT_U ? tile / 2 : tile;
    const long long ti = local / e.tiles_r, tr = local % e.tiles_r;
    sl.op = e.op;
    sl.l_first = e.l0 + ti * tl;
    sl.nl = (int)min((long long)tl, e.l1 - sl.l_first);
    sl.row0 = e.r0 + tr * rc;
    sl.nrows = skip ? 1 : (int)min((long long)rc, e.r1 - sl.row0);
    return skip ? 0u : (u32)sl.nl * (u32)pitch * 8u;
}

// Producer state kept in shared memory: the plan (instance, sequence) whose entries are cached.
struct ProdCache {
    int inst;
    u32 seq;
    int nentries;
    int cur;              // entry in `e`
    int rc, ur, cost, check_only;
    long long plan_items;
    int trace_first;      // the next item filled is this producer's first of the plan
    int split_small;      // the plan's level has fewer than SPLIT_MAX_CANDS candidates
    long long item0[ENTRY_CACHE];
    Entry e;
    InstArgs a;           // the instance's arguments (read once per plan)
};

__device__ __forceinline__ InstCtl *ctl_of(const Launch &L, int inst) { return (InstCtl *)__ldcg((const u64 *)&L.args[inst].ctl); }

// Every instance of the launch is finished (a batch: no instance pending and no slot searching).
__device__ __forceinline__ bool launch_done(const Launch &L, int lane) {
    if (L.batch) {
        bool d = true;
        if (lane == 0)
            d = ld_volatile(&L.batch->next) >= (u64)L.batch->count && *(volatile int *)&L.batch->live == 0;
        return __shfl_sync(FULL, d, 0);
    }
    bool all_done = true;
    for (int q = lane; q < L.ninst; q += 32)
        if (!(*(volatile u32 *)&ctl_of(L, q)->flags & CTL_DONE)) all_done = false;
    return __all_sync(FULL, all_done);
}

// The producer warp: claims items, fills slots, issues the tile copies and the L2 prefetches.
template <int TL>
__device__ void producer(const Launch &L, unsigned char *smem, u64 *tiles, int lane) {
    __shared__ ProdCache pc;
    const int S = L.stages;
    const long long tile_words = L.tile_bytes / 8;
    if (lane == 0) {
        pc.inst = -1;
        pc.seq = 0;
        pc.cur = -1;
    }
    __syncwarp();
    int inst = (int)(blockIdx.x % (unsigned)L.ninst);
    u64 k = 0;
    bool ended = false, optimistic = false;
    while (!ended) {
        const int s = (int)(k % (u64)S);
        Slot &sl = *slot_at(smem, s);
        if (k >= (u64)S) {
            bool ok = true;
            if (lane == 0) ok = mbar_wait_for(&sl.empty, (u32)(((k / S) - 1) & 1), EMPTY_WAIT_NS);
            ok = __shfl_sync(FULL, ok, 0);
            if (!ok) {
                if (lane == 0) atomicOr(&ctl_of(L, inst)->status, ST_TMA);
                ended = true;  // the slot may still be read: leave without filling it
                break;
            }
        }
        // claim an item from some instance.  After a successful claim the next one is
        // optimistic: the limit, the find key and the claim are issued together (one round
        // trip); after a failed one the producer looks before it takes, so idle polls do not
        // advance the counter.
        long long item = -1;
        u64 tag = 0, fk = NO_FIND;
        u32 ovf = 0;
        int tries = 0;
        u64 t_wait = 0, last_done = ~0ull;
        for (;;) {
            InstCtl *C = ctl_of(L, inst);
            u64 v = 0, lim = 0, f = NO_FIND;
            u32 stt = 0;
            if (lane == 0) {
                if (optimistic) {
                    lim = ld_volatile(&C->limit);
                    f = ld_volatile(&C->found_key);
                    stt = *(volatile const u32 *)&C->status;
                    v = atomicAdd(&C->claimed, 1ull);
                    if ((v >> SEQ_SHIFT) != (lim >> SEQ_SHIFT)) {  // a newer plan: its limit was released before it
                        __threadfence();
                        lim = ld_volatile(&C->limit);
                    }
                } else {
                    lim = ld_volatile(&C->limit);
                    const u64 cur = ld_volatile(&C->claimed);
                    v = cur;
                    if ((cur >> SEQ_SHIFT) == (lim >> SEQ_SHIFT) && cur < lim) {
                        f = ld_volatile(&C->found_key);
                        stt = *(volatile const u32 *)&C->status;
                        v = atomicAdd(&C->claimed, 1ull);
                        if ((v >> SEQ_SHIFT) != (lim >> SEQ_SHIFT)) {
                            __threadfence();
                            lim = ld_volatile(&C->limit);
                        }
                    }
                }
            }
            v = __shfl_sync(FULL, v, 0);
            lim = __shfl_sync(FULL, lim, 0);
            f = __shfl_sync(FULL, f, 0);
            if ((v >> SEQ_SHIFT) == (lim >> SEQ_SHIFT) && v < lim) {
                item = (long long)(v & ITEM_MASK);
                tag = v >> SEQ_SHIFT;
                fk = f;
                ovf = __shfl_sync(FULL, stt, 0) & ST_OVERFLOW;
                optimistic = true;
                break;
            }
            optimistic = false;
            // nothing to take from this instance now
            if (++tries < L.ninst) {
                inst = (inst + 1) % L.ninst;
                continue;
            }
            tries = 0;
            if (!L.persist || launch_done(L, lane)) {
                ended = true;
                break;
            }
            // wait for a new plan (some instance's level is finishing); give up without progress
            u64 d = 0;
            if (lane == 0) {
                for (int q = 0; q < L.ninst; ++q) {
                    InstCtl *Cq = ctl_of(L, q);
                    d += ld_volatile(&Cq->done) + ld_volatile(&Cq->limit);
                }
            }
            d = __shfl_sync(FULL, d, 0);
            const u64 now = globaltimer();
            if (d != last_done) {
                last_done = d;
                t_wait = now;
            } else if (now - t_wait > STALL_NS) {
                if (lane == 0) atomicOr(&C->status, ST_STALL);
                ended = true;
                break;
            }
            __nanosleep(256);
        }
        if (ended) break;
        InstCtl *C = ctl_of(L, inst);
        // the plan's arguments and entry starts (per instance and sequence)
        if (pc.inst != inst || pc.seq != (u32)tag) {
            __threadfence();  // the new plan was published before the claim counter this claim read
            constexpr int AW = sizeof(InstArgs) / 8;
            for (int w = lane; w < AW; w += 32)
                reinterpret_cast<u64 *>(&pc.a)[w] = __ldcg(reinterpret_cast<const u64 *>(L.args + inst) + w);
            __syncwarp();
            int nent = 0, rc = 1, ur = 1, cost = 0, chk = 0;
            long long pitems = 0;
            if (lane == 0) {
                nent = __ldcg(&C->plan.nentries);
                rc = __ldcg(&C->plan.right_chunk);
                ur = __ldcg(&C->plan.unary_rows);
                cost = __ldcg(&C->plan.cost);
                chk = __ldcg(&C->plan.check_only);
                pitems = __ldcg(&C->plan.items);
            }
            nent = __shfl_sync(FULL, nent, 0);
            for (int e = lane; e < nent && e < ENTRY_CACHE; e += 32) pc.item0[e] = __ldcg(&pc.a.entries[e].item0);
            if (lane == 0) {
                // rows of the finished levels were written through the generic proxy; the tile
                // copies read them through the async proxy
                fence_proxy_async_global();
                pc.inst = inst;
                pc.seq = (u32)tag;
                pc.nentries = nent;
                pc.cur = -1;
                pc.rc = rc;
                pc.ur = ur;
                pc.cost = cost;
                pc.check_only = chk;
                pc.plan_items = pitems;
                pc.split_small = __ldcg(&C->plan.cand) < SPLIT_MAX_CANDS;
                pc.trace_first = pc.a.level_ns != nullptr;
                if (pc.trace_first) atomicCAS(pc.a.level_ns + (u64)cost * LEVEL_TRACE + LT_CLAIMED, 0ull, globaltimer());
            }
            __syncwarp();
        }
        // the entry holding the item: the last one whose item0 <= item
        int lo = 0, hi = pc.nentries - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            const long long m0 = mid < ENTRY_CACHE ? pc.item0[mid] : __ldcg(&pc.a.entries[mid].item0);
            if (m0 <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        if (pc.cur != lo) {
            constexpr int W = sizeof(Entry) / 8;
            const u64 *src = reinterpret_cast<const u64 *>(pc.a.entries + lo);
            if (lane < W) reinterpret_cast<u64 *>(&pc.e)[lane] = __ldcg(src + lane);
            __syncwarp();
            if (lane == 0) pc.cur = lo;
            __syncwarp();
        }
        // skip rule: a find at or before this entry's block (or any find, find_first) in this level
        const bool found_here = pc.a.stop_at_found && fk != NO_FIND && (int)(fk >> 32) == pc.cost;
        const bool skip = found_here && (pc.a.find_first || pc.e.pos >= (int)(u32)fk);
        // the same rule for the items of this level still in this CTA's slots: their remaining
        // rows are skipped (the slot the producer is about to fill is not in flight)
        if (found_here && lane < S && lane != s) {
            Slot &o = *slot_at(smem, lane);
            if (*(volatile int *)&o.kind != 0 && o.inst == inst && o.cost == pc.cost &&
                (pc.a.find_first || o.pos >= (int)(u32)fk))
                *(volatile int *)&o.stop = 1;
        }
        {
            constexpr int AW = sizeof(InstArgs) / 8;
            for (int w = lane; w < AW; w += 32)
                reinterpret_cast<u64 *>(&sl.args)[w] = reinterpret_cast<const u64 *>(&pc.a)[w];
            __syncwarp();
        }
        if (lane == 0) {
            const u32 bytes = fill_slot(sl, inst, pc.e, item, L.tile, pc.rc, pc.ur, pc.cost, pc.check_only,
                                        pc.plan_items, skip, pc.a.pitch);
            sl.trace_first = pc.trace_first;
            sl.overflowed = ovf ? 1 : 0;
            // a small level's rows are split into one unit per left row / unary operator, so
            // more warps share its few rows (one warp's pass over a whole row is what such a
            // level costs)
            int split = 1;
            if (!skip && pc.split_small) split = sl.kind == ENT_UNARY ? __popc((unsigned)sl.op) : sl.nl;
            sl.split = max(1, split);
            sl.units = sl.nrows * sl.split;
            pc.trace_first = 0;
            if (!skip) {
                const u64 pitch = (u64)pc.a.pitch;
                const u64 rows_bytes = (u64)sl.nrows * pitch * 8;
                if (rows_bytes > 0 && rows_bytes < (1ull << 31))
                    prefetch_l2(pc.a.cache + (u64)sl.row0 * pitch, (u32)rows_bytes);
            }
            if (bytes) {
                fence_proxy_async();
                mbar_expect_tx(&sl.full, bytes);
                bulk_g2s(tiles + (u64)s * tile_words, pc.a.cache + (u64)sl.l_first * pc.a.pitch, bytes, &sl.full);
            } else {
                mbar_arrive(&sl.full);
            }
        }
        __syncwarp();
        ++k;
    }
    // the end: every consumer sees a slot of kind 0 (the slot after the last one filled)
    const int s = (int)(k % (u64)S);
    Slot &sl = *slot_at(smem, s);
    if (k >= (u64)S && lane == 0) mbar_wait_for(&sl.empty, (u32)(((k / S) - 1) & 1), EMPTY_WAIT_NS);
    if (lane == 0) {
        sl.kind = 0;
        mbar_arrive(&sl.full);
    }
    __syncwarp();
}

// The units of one slot a consumer warp takes, until the slot has none left: a unit is one row
// of the item, or at a small level (split > 1) one left row of the tile against one right row,
// or one unary operator on one source row.  Returns SLOT_CLOSE when this warp finished the
// level's last item, else SLOT_NEXT; closing the level (with the slot's arguments, before the
// slot is released) is the caller's.
enum { SLOT_NEXT = 0, SLOT_CLOSE = 1 };
template <int TL, int HK>
__device__ __forceinline__ int take_rows(Slot &sl, int kind, const ulonglong2 *tile, int lane) {
    const InstArgs &A = sl.args;
    InstCtl *C = A.ctl;
    int out = SLOT_NEXT;
    for (;;) {
        unsigned idx = 0;
        if (lane == 0) idx = atomicAdd(&sl.next_row, 1u);
        idx = __shfl_sync(FULL, idx, 0);
        if ((int)idx >= sl.units) break;
        if (idx == 0 && sl.trace_first && lane == 0)
            atomicCAS(A.level_ns + (u64)sl.cost * LEVEL_TRACE + LT_STARTED, 0ull, globaltimer());
        if (!*(volatile int *)&sl.stop) {
            // a unit is a row, or with split one left row (binary) or one operator (unary) of it
            const int split = sl.split, part = (int)idx % split;
            const long long r = sl.row0 + (int)idx / split;
            const ulonglong2 *rp = reinterpret_cast<const ulonglong2 *>(A.cache + (u64)r * A.pitch);
            if (kind == ENT_UNARY) {
                int mask = sl.op;
                for (int q = 0; q < part && split > 1; ++q) mask &= mask - 1;  // the part-th operator
                unary_row<HK>(A, C, sl, split > 1 ? (mask & -mask) : mask, rp, r, lane);
            } else {
                const int nch = A.pitch >> 1;
                const ulonglong2 *t0 = split > 1 ? tile + (u64)part * (u64)nch : tile;
                const int nl = split > 1 ? 1 : sl.nl;
                const long long lf = sl.l_first + (split > 1 ? part : 0);
                if (kind == ENT_ANDOR)
                    binary_row<OP_ANDOR_CLASS, TL, HK>(A, C, sl, t0, nl, lf, rp, r, lane);
                else
                    binary_row<OP_U, TL, HK>(A, C, sl, t0, nl, lf, rp, r, lane);
            }
        }
        unsigned d = 0;
        __threadfence_block();  // this row's evals count is in before the row counts as done
        if (lane == 0) d = atomicAdd(&sl.rows_done, 1u);
        d = __shfl_sync(FULL, d, 0);
        if ((int)d + 1 == sl.units) {  // the item is done
            u64 dd = 0;
            if (lane == 0) {
                const unsigned ev = atomicAdd(&sl.evals, 0u);
                if (ev) atomicAdd(&C->evaluated, (u64)ev);
                __threadfence();
                dd = atomicAdd(&C->done, 1ull);
            }
            dd = __shfl_sync(FULL, dd, 0);
            if ((long long)dd + 1 == sl.plan_items) out = SLOT_CLOSE;
        }
    }
    return out;
}

// A consumer warp: takes the rows of the slots in order until the producer's end slot; the
// warp that finishes a level's last item closes the level (and plans the next one).
template <int TL, int HK>
__device__ void consumer(const Launch &L, unsigned char *smem, const u64 *tiles, int lane) {
    const int S = L.stages;
    const long long tile_words = L.tile_bytes / 8;
    for (u64 k = 0;; ++k) {
        const int s = (int)(k % (u64)S);
        Slot &sl = *slot_at(smem, s);
        bool ok = true;
        if (lane == 0) ok = mbar_wait_for(&sl.full, (u32)((k / S) & 1), PIPE_WAIT_NS);
        ok = __shfl_sync(FULL, ok, 0);
        if (!ok) {
            if (lane == 0) atomicOr(&ctl_of(L, 0)->status, ST_TMA);
            return;
        }
        const int kind = *(volatile int *)&sl.kind;
        if (kind == 0) return;
        const ulonglong2 *tile = reinterpret_cast<const ulonglong2 *>(tiles + (u64)s * tile_words);
        const int got = take_rows<TL, HK>(sl, kind, tile, lane);
        int recycle = -1;  // a batch slot whose instance's search ended in this warp
        if (got == SLOT_CLOSE) {  // the slot's arguments are read before the slot is released
            const bool ended = close_level(sl.args, sl.args.ctl, L.persist != 0, lane);
            if (ended && L.batch) recycle = sl.inst;
        }
        if (lane == 0) mbar_arrive(&sl.empty);
        __syncwarp();
        if (recycle >= 0) next_instance<HK>(*L.batch, recycle, true, lane);
    }
}

}  // namespace

// ---------------------------------------------------------------- kernels
namespace {

__device__ __forceinline__ size_t slots_bytes(int S) { return ((size_t)S * sizeof(Slot) + 127) & ~(size_t)127; }

template <int TL, int HK>
__global__ void __launch_bounds__(LEVEL_THREADS, 1) level_kernel(const Launch *__restrict__ Lp) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ Launch L;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        L = *Lp;
        for (int s = 0; s < L.stages; ++s) {
            Slot &sl = *slot_at(smem, s);
            mbar_init(&sl.full, 1);
            mbar_init(&sl.empty, NCONS);
        }
        fence_mbar_init();
    }
    __syncthreads();
    u64 *tiles = reinterpret_cast<u64 *>(smem + slots_bytes(L.stages));
    if (warp == 0)
        producer<TL>(L, smem, tiles, lane);
    else
        consumer<TL, HK>(L, smem, tiles, lane);
}

// A batch's first instances: block s sets slot s up (one warp per slot).
template <int HK>
__global__ void batch_start_kernel(BatchDev *__restrict__ B) {
    if (threadIdx.x >= 32) return;
    next_instance<HK>(*B, (int)blockIdx.x, false, threadIdx.x & 31);
}

// The first plan of each instance: the letters (cost c1, rows [0, nalpha)) form the level
// that has just ended.  One warp per instance; the host has set plan.cost = c1, row_count =
// nalpha, the level starts to 0 and found_key to NO_FIND.
__global__ void first_plan_kernel(const InstArgs *__restrict__ args, int open) {
    const InstArgs &A = args[blockIdx.x];
    const int lane = threadIdx.x & 31;
    if (threadIdx.x >= 32) return;
    if (lane == 0) A.ctl->t_start = globaltimer();
    close_level(A, A.ctl, open != 0, lane);
}

// Plans level `cost` (the levels below are complete) and publishes the plan closed.
__global__ void plan_only_kernel(const InstArgs *__restrict__ args, int cost) {
    const InstArgs &A = *args;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x >= 32) return;
    plan_level(A, A.ctl, cost, lane);
    if (A.plan_flags & PLAN_LEARNED) score_plan(A, A.ctl, lane);
    if (lane == 0) publish(A.ctl, __ldcg(&A.ctl->plan.items), false);
}

// Letters: register rows [0, nalpha) in the hash set (duplicate letters stay rows,
// as the reference stores every letter, ltli6463.cu:1134, :1189-1190).  One warp per letter.
template <int HK>
__global__ void insert_letters_kernel(const InstArgs *__restrict__ pA, int nalpha) {
    const InstArgs &A = *pA;
    const int lane = threadIdx.x & 31, j = threadIdx.x >> 5;  // warp j: letter j
    const int nch = A.pitch >> 1;
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
            const u64 p0 = 2 * c < A.npos ? 1ull : 0ull, p1 = 2 * c + 1 < A.npos ? 1ull : 0ull;
            pm |= pmiss2(w.x, w.y, p0, p1);
            nh |= nhit2(w.x, w.y, p0, p1);
        }
        if (A.lstats)  // every letter is a stored row of the letter level
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
        case OP_NEG:
        case OP_X:
        case OP_F:
        case OP_G: w = unary_word(op, x, m); break;
        case OP_AND: w = x & y; break;
        case OP_OR: w = x | y; break;
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
// operators are the enumerator's own.
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
            v = unary_word(op, stack[(u64)(sp - 1) * n + t], m);
            --sp;
        } else {
            const u64 y = stack[(u64)(sp - 1) * n + t], x = stack[(u64)(sp - 2) * n + t];
            v = op == OP_U ? until_bits(x, y) : op == OP_AND ? (x & y) : (x | y);
            sp -= 2;
        }
        stack[(u64)sp * n + t] = v;
        ++sp;
    }
    out[t] = stack[t];
}

// The dynamic shared-memory limit is a per-device function attribute: each device keeps the
// largest size enabled on it so far.
template <int TL, int HK>
cudaError_t smem_attr(size_t smem) {
    constexpr int MAX_DEVICES = 64;
    static std::atomic<long long> attr_set[MAX_DEVICES];
    if (smem <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < MAX_DEVICES && (long long)smem <= attr_set[dev].load()) return cudaSuccess;
    e = cudaFuncSetAttribute(level_kernel<TL, HK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && dev >= 0 && dev < MAX_DEVICES) {
        long long cur = attr_set[dev].load();
        while (cur < (long long)smem && !attr_set[dev].compare_exchange_weak(cur, (long long)smem)) {
        }
    }
    return e;
}

template <int TL, int HK>
cudaError_t launch_tl(const Launch &h, const Launch *d, int grid, cudaStream_t s) {
    const size_t smem = level_kernel_smem(h.stages, h.tile_bytes);
    cudaError_t e = smem_attr<TL, HK>(smem);
    if (e != cudaSuccess) return e;
    level_kernel<TL, HK><<<grid, LEVEL_THREADS, smem, s>>>(d);
    return cudaGetLastError();
}

template <int TL, int HK>
int occupancy_tl(size_t smem) {
    if (smem_attr<TL, HK>(smem) != cudaSuccess) return 0;
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, level_kernel<TL, HK>, LEVEL_THREADS, smem) ==
                   cudaSuccess
               ? n
               : 0;
}

template <int HK>
cudaError_t launch_hk(const Launch &h, const Launch *d, int grid, cudaStream_t s) {
    return h.tile == 2   ? launch_tl<2, HK>(h, d, grid, s)
           : h.tile == 4 ? launch_tl<4, HK>(h, d, grid, s)
                         : launch_tl<8, HK>(h, d, grid, s);
}

}  // namespace

size_t level_kernel_smem(int stages, long long tile_bytes) {
    return (((size_t)stages * sizeof(Slot) + 127) & ~(size_t)127) + (size_t)stages * (size_t)tile_bytes;
}

cudaError_t launch_levels(const Launch &h, const Launch *d, int grid, int hk, cudaStream_t s) {
    return hk == 1 ? launch_hk<1>(h, d, grid, s) : launch_hk<0>(h, d, grid, s);
}

int level_kernel_ctas_per_sm(int hk, size_t smem) {
    // every tile instance has the same resource use up to its registers; ask the 8-row one
    return hk == 1 ? occupancy_tl<8, 1>(smem) : occupancy_tl<8, 0>(smem);
}

cudaError_t launch_first_plan(const InstArgs *d, int ninst, int open, cudaStream_t s) {
    first_plan_kernel<<<ninst, 32, 0, s>>>(d, open);
    return cudaGetLastError();
}

cudaError_t launch_batch_start(BatchDev *d, int nslots, int hk, cudaStream_t s) {
    if (hk == 1)
        batch_start_kernel<1><<<nslots, 32, 0, s>>>(d);
    else
        batch_start_kernel<0><<<nslots, 32, 0, s>>>(d);
    return cudaGetLastError();
}

cudaError_t launch_plan_level(const InstArgs *d, int cost, cudaStream_t s) {
    plan_only_kernel<<<1, 32, 0, s>>>(d, cost);
    return cudaGetLastError();
}

cudaError_t launch_insert_letters(const InstArgs *d, int nalpha, int hk, cudaStream_t s) {
    const int threads = 32 * (nalpha > 0 ? nalpha : 1);
    if (hk == 1)
        insert_letters_kernel<1><<<1, threads, 0, s>>>(d, nalpha);
    else
        insert_letters_kernel<0><<<1, threads, 0, s>>>(d, nalpha);
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

cudaError_t launch_eval_formula(const int *prog, int len, const u64 *atoms, const u64 *lenmask, int n, u64 *stack,
                                u64 *out, cudaStream_t s) {
    eval_formula_kernel<<<(n + 127) / 128, 128, 0, s>>>(prog, len, atoms, lenmask, n, stack, out);
    return cudaGetLastError();
}

}  // namespace ltlg
