// K4: per-partition bucket sort and pilot search; persistent warps, one
// partition per warp at a time, taken from a shared work queue.
//
// Replaces sort_sum.comp:141-226 (bucket histogram, descending-size order,
// in-partition offsets), redistribute_keys.comp:21-53 (bucket order inside the
// partition) and search.comp:31-175 (the pilot search).
//
// Order and result follow the reference exactly:
//   * buckets are searched by descending size, and by descending bucket index
//     among equal sizes (sort_sum.comp:156-172, search.comp:145-166);
//   * for each bucket the pilot counter k starts at 0; k is rejected when two
//     keys of the bucket hash to the same slot (search.comp:44-70); otherwise
//     the smallest offset o in [0, ps) whose slots (h_i + o) mod ps are all free
//     is taken (search.comp:72-103 under lockstep execution), the slots are
//     marked, and pilot = o + ps * k (search.comp:122);
//   * pilots are stored bucket-major at pilots[b * partitions + p]
//     (search.comp:170-174); empty buckets get 0.
//
// Work queue: every warp takes the next global partition from one counter, so
// partitions of very different cost (and of different key sets in a batched
// build) spread over the SMs without CTA-level tail imbalance.
//
// Offset search: the occupancy bitmap is stored twice in a row (bits [ps, 2 ps)
// repeat bits [0, ps)), so the 32 slots (h + o) mod ps, o in [w, w + 32), are the
// bits [h + w, h + w + 32) of the doubled bitmap for any slot h < ps and w < ps,
// read with two loads and one funnel shift.  Lane L tests offsets [w, w + 32),
// w = w0 + 32 L, by OR-ing the windows of all keys of the bucket; a warp covers
// 1024 offsets per round and the first lane with a free window holds the
// smallest valid offset.  Because w is a multiple of 32, the word index of a
// window is (h >> 5) + (w >> 5) and its bit shift is h & 31 for every lane.
//
// Buckets of at most 32 keys (nearly all of them) keep one key per lane in
// registers and test collisions with __match_any_sync; for at most 8 keys the
// offset search also keeps every slot in registers (as 4 or 8 slots, the unused
// ones repeating slot 0), for 9..32 keys it reads them from shared memory four at
// a time.  Larger buckets read their keys from the
// bucket-ordered copy in global memory and stage their slots in shared memory.
#include "kernels.cuh"

namespace phobicb200 {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kHsWords = 260;  // packed slots of up to 256 keys, padded to a multiple of 4

// Occupancy bitmap of a partition of at most cap slots, stored twice in a row
// (bits [ps, 2 ps) repeat bits [0, ps)) plus one spare word.
__host__ __device__ __forceinline__ uint32_t occ_words(uint32_t cap) { return (2 * cap + 31) / 32 + 2; }
// Collision scratch of large buckets: one bit per slot.
__host__ __device__ __forceinline__ uint32_t scr_words(uint32_t cap) { return (cap + 31) / 32 + 1; }
__host__ __device__ __forceinline__ uint32_t half_words(uint32_t B) { return (B + 1) / 2; }
// Words of the bitmap: the doubled bitmap plus room for every read of the
// register-path offset search, which reads, for a slot h < ps and lane L in round
// r < ceil(ps / 1024), words (h >> 5) + L + 32 r and the one after it, dead lanes
// included; the bound covers it for every ps <= cap.
__host__ __device__ __forceinline__ uint32_t bitmap_words(uint32_t cap) {
    uint32_t reach = (cap - 1) / 32 + 32 * ((cap + 1023) / 1024) + 2;
    return reach > occ_words(cap) ? reach : occ_words(cap);
}

// Per-warp shared memory, in 32-bit words.  Every warp's region starts on a
// 16-byte boundary (its size is rounded up to 4 words) and the union comes
// first, so hs is 16-byte aligned for the 128-bit slot loads:
//   union of
//     prep phase:    cur u16[B] bucket cursors, binPos u16[256], binKey u16[256]
//     search phase:  hs [260] packed slots, scr [SW] collision scratch of large buckets
//   cnt   u16[B]     bucket sizes
//   sched [B]        search schedule, in search order: start | bucket << 16
//   occ   [OW]       occupied slots, bits [ps, 2 ps) mirror [0, ps)
__host__ __device__ __forceinline__ size_t union_words(uint32_t B, uint32_t cap) {
    size_t prep = (size_t)half_words(B) + 256, search = kHsWords + scr_words(cap);
    return prep > search ? prep : search;
}

__host__ __device__ __forceinline__ size_t warp_words(uint32_t B, uint32_t cap) {
    size_t w = union_words(B, cap) + half_words(B) + (size_t)B + (size_t)bitmap_words(cap);
    return (w + 3) & ~size_t(3);
}

struct WarpSmem {
    uint32_t *cur32, *binPos, *binKey;  // packed u16 pairs (prep phase)
    uint32_t *hs, *scr;                 // search phase
    uint32_t *cnt32;                    // packed u16 pairs
    uint32_t *sched;
    uint32_t *occ;
    uint32_t occ_lo, occ_hi;  // shared-space byte bounds of the bitmap (checked build)
};

__device__ __forceinline__ WarpSmem carve(uint32_t *w, uint32_t B, uint32_t cap) {
    WarpSmem m;
    m.cur32 = w;
    m.binPos = w + half_words(B);
    m.binKey = m.binPos + 128;
    m.hs = w;
    m.scr = w + kHsWords;
    m.cnt32 = w + union_words(B, cap);
    m.sched = m.cnt32 + half_words(B);
    m.occ = m.sched + B;
    m.occ_lo = (uint32_t)__cvta_generic_to_shared(m.occ);
    m.occ_hi = m.occ_lo + 4 * bitmap_words(cap);
    return m;
}

__device__ __forceinline__ uint32_t half_get(const uint32_t *w, uint32_t b) { return (w[b >> 1] >> ((b & 1) << 4)) & 0xFFFFu; }
// Adds v to the u16 entry b of a packed array (no entry may exceed 0xFFFF).
__device__ __forceinline__ void half_add_n(uint32_t *w, uint32_t b, uint32_t v) { atomicAdd(&w[b >> 1], v << ((b & 1) << 4)); }
__device__ __forceinline__ uint32_t half_add(uint32_t *w, uint32_t b) {
    uint32_t sh = (b & 1) << 4;
    return (atomicAdd(&w[b >> 1], 1u << sh) >> sh) & 0xFFFFu;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(kFullMask, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

__device__ __forceinline__ void mark(uint32_t *occ, uint32_t q, uint32_t ps) {
    atomicOr(&occ[q >> 5], 1u << (q & 31));
    const uint32_t m = q + ps;
    atomicOr(&occ[m >> 5], 1u << (m & 31));
}

__device__ __forceinline__ uint32_t lds32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}
__device__ __forceinline__ uint32_t lds32_next(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1+4];" : "=r"(v) : "r"(addr));
    return v;
}
// The 32-bit window starting `sh` bits into the bitmap word at byte address `addr`;
// in the checked build the two words must lie inside [lo, hi).
__device__ __forceinline__ uint32_t window_at(uint32_t addr, uint32_t sh, uint32_t lo, uint32_t hi) {
    if (!PHB_CHECK(addr >= lo && addr + 8 <= hi)) return kFullMask;
    return __funnelshift_r(lds32(addr), lds32_next(addr), sh);
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
    return v;
}

// A slot h as the offset search reads it: the byte offset of its bitmap word,
// 4 * (h >> 5), shifted left by 5, with the bit position h & 31 in the low bits.
// The funnel shift only looks at the low 5 bits, so one word serves both uses.
__device__ __forceinline__ uint32_t pack_slot(uint32_t h) { return ((h >> 5) << 7) | (h & 31); }
__device__ __forceinline__ uint32_t unpack_slot(uint32_t v) { return ((v >> 7) << 5) | (v & 31); }

// Smallest free offset in rounds of 1024 (see the offset search above).  hs holds
// the s packed slots of the bucket, 16-byte aligned, padded to a multiple of 4
// with copies of slot 0 (OR is idempotent); each group of 4 is one broadcast
// 128-bit load.  A round stops early once every lane's window holds an occupied
// slot.  The bitmap is addressed through 32-bit shared-memory addresses.
__device__ __forceinline__ uint32_t first_free_offset(const uint32_t *occ, const uint32_t *hs, uint32_t s,
                                                      uint32_t ps, int lane, uint32_t lo, uint32_t hi) {
    const uint32_t occ_sa = (uint32_t)__cvta_generic_to_shared(occ);
    const uint32_t hs_sa = (uint32_t)__cvta_generic_to_shared(hs);
    for (uint32_t w0 = 0; w0 < ps; w0 += 1024) {
        const uint32_t w = w0 + 32 * lane;
        const bool live = w < ps;
        const uint32_t base = occ_sa + (live ? (w >> 3) : 0u);
        uint32_t bad = live ? 0u : kFullMask;
        for (uint32_t i = 0; i < s; i += 4) {
            const uint4 v = lds128(hs_sa + 4 * i);
            const uint32_t a0 = base + (v.x >> 5), a1 = base + (v.y >> 5);
            const uint32_t a2 = base + (v.z >> 5), a3 = base + (v.w >> 5);
            bad |= window_at(a0, v.x, lo, hi) | window_at(a1, v.y, lo, hi);
            bad |= window_at(a2, v.z, lo, hi) | window_at(a3, v.w, lo, hi);
            if (__all_sync(kFullMask, bad == kFullMask)) break;
        }
        uint32_t valid = ~bad;
        if (live && ps - w < 32) valid &= (1u << (ps - w)) - 1u;
        const uint32_t ball = __ballot_sync(kFullMask, valid != 0);
        if (ball) {
            const int f = __ffs(ball) - 1;
            return w0 + 32 * f + __ffs(__shfl_sync(kFullMask, valid, f)) - 1;
        }
    }
    return kNone;
}

// The same search for a bucket of at most K <= 8 keys, with the packed slots in
// registers: hp is this lane's packed slot, lanes >= the bucket size hold slot 0's.
// Each key's bitmap address is formed once per call (occ + (h >> 5) words); a round
// adds the lane's window offset.  K == 8 tests the second half only when some live
// window is still open after the first four keys.  Dead lanes (w >= ps) read at
// offset 0, inside the bitmap, and count as fully occupied.
template <int K>
__device__ __forceinline__ uint32_t first_free_offset_reg(const uint32_t *occ, uint32_t hp, uint32_t ps, int lane,
                                                          uint32_t blo, uint32_t bhi) {
    const uint32_t occ_sa = (uint32_t)__cvta_generic_to_shared(occ);
    uint32_t v[K], hb[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        v[i] = __shfl_sync(kFullMask, hp, i);
        hb[i] = occ_sa + (v[i] >> 5);
    }
    for (uint32_t w0 = 0; w0 < ps; w0 += 1024) {
        const uint32_t w = w0 + 32 * lane;
        const bool live = w < ps;
        const uint32_t lo = live ? (w >> 3) : 0u;
        uint32_t bad = 0;
#pragma unroll
        for (int i = 0; i < (K < 4 ? K : 4); i++) bad |= window_at(hb[i] + lo, v[i], blo, bhi);
        if (K == 8) {
            if (!__all_sync(kFullMask, bad == kFullMask || !live)) {
#pragma unroll
                for (int i = 4; i < K; i++) bad |= window_at(hb[i] + lo, v[i], blo, bhi);
            }
        }
        uint32_t valid = live ? ~bad : 0u;
        if (live && ps - w < 32) valid &= (1u << (ps - w)) - 1u;
        const uint32_t ball = __ballot_sync(kFullMask, valid != 0);
        if (ball) {
            const int f = __ffs(ball) - 1;
            return w0 + 32 * f + __ffs(__shfl_sync(kFullMask, valid, f)) - 1;
        }
    }
    return kNone;
}

template <int OFF>
__device__ __forceinline__ uint32_t lds32_at(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1+%2];" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

// Round R (offsets [1024 R, 1024 R + 1024)) of first_free_offset_unr: true when
// some lane's window holds a free offset, which is written to *o.
template <int K, int R>
__device__ __forceinline__ bool scan_round(const uint32_t (&hb)[K], const uint32_t (&v)[K], uint32_t ps, int lane,
                                           uint32_t *o, uint32_t blo, uint32_t bhi) {
    // Offsets of this lane's window below ps, as a mask (clamped funnel shift: n >= 32 gives all ones).
    const int n = (int)ps - (int)(1024 * R) - 32 * lane;
    uint32_t bad = ~__funnelshift_lc(kFullMask, 0u, (uint32_t)max(n, 0));
#pragma unroll
    for (int i = 0; i < (K < 4 ? K : 4); i++)
        bad |= PHB_CHECK(hb[i] + 128 * R >= blo && hb[i] + 128 * R + 8 <= bhi)
                   ? __funnelshift_r(lds32_at<128 * R>(hb[i]), lds32_at<128 * R + 4>(hb[i]), v[i])
                   : kFullMask;
    if (K == 8) {
        if (!__all_sync(kFullMask, bad == kFullMask)) {
#pragma unroll
            for (int i = 4; i < K; i++)
                bad |= PHB_CHECK(hb[i] + 128 * R >= blo && hb[i] + 128 * R + 8 <= bhi)
                           ? __funnelshift_r(lds32_at<128 * R>(hb[i]), lds32_at<128 * R + 4>(hb[i]), v[i])
                           : kFullMask;
        }
    }
    const uint32_t ball = __ballot_sync(kFullMask, bad != kFullMask);
    if (!ball) return false;
    const int f = __ffs(ball) - 1;
    *o = 1024u * R + 32u * f + __ffs(~__shfl_sync(kFullMask, bad, f)) - 1;
    return true;
}

// first_free_offset_reg for ps <= 3072: the (at most three) rounds unrolled, each
// key's window address formed once per call with the lane's word offset included,
// so a round reads at a constant 128 R bytes further.  Dead lanes (offsets >= ps)
// read inside the padded bitmap (bitmap_words) and are masked.
template <int K>
__device__ __forceinline__ uint32_t first_free_offset_unr(const uint32_t *occ, uint32_t hp, uint32_t ps,
                                                          uint32_t rounds, int lane, uint32_t blo, uint32_t bhi) {
    const uint32_t lane_sa = (uint32_t)__cvta_generic_to_shared(occ) + 4u * lane;
    uint32_t v[K], hb[K];
#pragma unroll
    for (int i = 0; i < K; i++) {
        v[i] = __shfl_sync(kFullMask, hp, i);
        hb[i] = lane_sa + (v[i] >> 5);
    }
    uint32_t o = kNone;
    if (scan_round<K, 0>(hb, v, ps, lane, &o, blo, bhi)) return o;
    if (rounds > 1 && scan_round<K, 1>(hb, v, ps, lane, &o, blo, bhi)) return o;
    if (rounds > 2 && scan_round<K, 2>(hb, v, ps, lane, &o, blo, bhi)) return o;
    return kNone;
}

// Whether two keys of a bucket of s <= 32 keys (key `lane` in L) are identical.
// Reached only when a bucket's pilot counter gets to kDupCheckAt, so it is kept
// out of line, away from the instructions of the search loop.
__device__ __noinline__ bool has_duplicate_key(uint2 L, uint32_t s, int lane) {
    bool d = false;
    for (uint32_t t = 0; t + 1 < s; t++) {
        uint32_t x = __shfl_sync(kFullMask, L.x, t), y = __shfl_sync(kFullMask, L.y, t);
        d |= lane < (int)s && lane > (int)t && L.x == x && L.y == y;
    }
    return __any_sync(kFullMask, d);
}

// Marks slot q (and its mirror q + ps) when `on`; predicated shared-memory reductions, so
// the lanes of a bucket mark without a divergent branch.
__device__ __forceinline__ void mark_if(uint32_t *occ, uint32_t q, uint32_t ps, bool on) {
    const uint32_t m = q + ps;
    const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(occ + (q >> 5)), a1 =
                           (uint32_t)__cvta_generic_to_shared(occ + (m >> 5));
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
        "@p red.shared.or.b32 [%0], %1;\n\t@p red.shared.or.b32 [%2], %3;\n\t}" ::"r"(a0),
        "r"(1u << (q & 31)), "r"(a1), "r"(1u << (m & 31)), "r"((uint32_t)on)
        : "memory");
}

// A bucket of at most S keys (S = 4 or 8) in a partition of at most 3072 slots: the warp
// hashes 32 / S pilot counters at once (lane t * S + i holds key i under counter k0 + t; lanes
// past the bucket hold key 0, the padding the scan expects) and tests them in counter order, so
// a counter that fails costs no new hash or collision test.  Same result as trying
// k = 0, 1, 2, ... one at a time (search.comp:105-124).  With MARK the slots are marked and
// *pilot written; without, nothing is marked and the bucket pipeline gets the counter, the
// offset and (lanes < s) the lane's slot in *k_out, *o_out, *q_out.
template <int S, bool MARK = true>
__device__ __forceinline__ uint32_t place_batched(const WarpSmem &ws, uint2 L, uint32_t s, uint32_t ps, FastMod fm,
                                                  uint32_t k_lim, uint32_t rounds, int lane, uint32_t *pilot,
                                                  uint32_t *k_out = nullptr, uint32_t *o_out = nullptr,
                                                  uint32_t *q_out = nullptr) {
    constexpr int G = 32 / S;
    constexpr uint32_t kGroupMask = (1u << S) - 1u;
    const int t = lane / S, i = lane % S;
    const bool key = i < (int)s;
    const uint32_t lx = __shfl_sync(kFullMask, L.x, key ? i : 0), ly = __shfl_sync(kFullMask, L.y, key ? i : 0);
    const int pick = lane < (int)s ? lane : 0;  // the key whose slot this lane passes to the scan
    const bool mine = lane < (int)s;
    for (uint32_t k0 = 0;; k0 += G) {
        const uint32_t hk = fm.mod(pilot_hash(lx, ly, k0 + (uint32_t)t));
        // Two keys of one counter on one slot: the counter rides above the slot (slots < 2^16).
        uint32_t coll = 0;
        if (s > 1) {
            const uint32_t v = key ? (hk | ((uint32_t)t << 24)) : (0x80000000u | (uint32_t)lane);
            const uint32_t m = __match_any_sync(kFullMask, v);
            coll = __ballot_sync(kFullMask, key && (m & (m - 1)) != 0);
        }
        const uint32_t pk = pack_slot(hk);
#pragma unroll 1
        for (int u = 0; u < G; u++) {
            const uint32_t k = k0 + (uint32_t)u;
            if (k >= k_lim) return PHOBIC_ERR_SEARCH_LIMIT;
            if (k == kDupCheckAt && s > 1 && has_duplicate_key(L, s, lane)) return PHOBIC_ERR_DUPLICATE_KEY;
            if ((coll >> (u * S)) & kGroupMask) continue;
            const uint32_t hp = __shfl_sync(kFullMask, pk, u * S + pick);
            const uint32_t o = first_free_offset_unr<S>(ws.occ, hp, ps, rounds, lane, ws.occ_lo, ws.occ_hi);
            if (o == kNone) continue;
            uint32_t q = __shfl_sync(kFullMask, hk, u * S + pick) + o;
            q = q >= ps ? q - ps : q;
            if constexpr (MARK) {
                mark_if(ws.occ, q, ps, mine && PHB_CHECK(!mine || q < ps));
                __syncwarp();
                *pilot = o + ps * k;
            } else {
                *k_out = k;
                *o_out = o;
                *q_out = q;
            }
            return PHOBIC_OK;
        }
    }
}

// One bucket of at most 32 keys; key `lane` in L.  Returns a status code.
__device__ __forceinline__ uint32_t place_small(const WarpSmem &ws, uint2 L, uint32_t s, uint32_t ps, FastMod fm,
                                                uint32_t k_lim, uint32_t rounds, int lane, uint32_t *pilot) {
    const bool mine = lane < (int)s;
    const uint32_t padded = (s + 3) & ~3u;
    // Every lane hashes (no divergent branch); lanes past the bucket take distinct
    // out-of-range values, so they never collide.  The hash of counter k + 1 is formed
    // while counter k is tested: the two dependency chains overlap.
    uint32_t hk_next = fm.mod(pilot_hash(L.x, L.y, 0u));
    for (uint32_t k = 0; k < k_lim; k++) {
        if (k == kDupCheckAt && s > 1 && has_duplicate_key(L, s, lane)) return PHOBIC_ERR_DUPLICATE_KEY;
        const uint32_t hk = hk_next;
        hk_next = fm.mod(pilot_hash(L.x, L.y, k + 1));
        const uint32_t h = mine ? hk : (0x80000000u | lane);
        if (s > 1) {
            uint32_t m = __match_any_sync(kFullMask, h);
            if (__any_sync(kFullMask, mine && (m & (m - 1)) != 0)) continue;
        }
        const uint32_t hp = pack_slot(__shfl_sync(kFullMask, h, mine ? lane : 0));
        uint32_t o;  // buckets of at most 8 keys with at most three rounds go to place_batched
        if (s <= 4) o = first_free_offset_reg<4>(ws.occ, hp, ps, lane, ws.occ_lo, ws.occ_hi);
        else if (s <= 8) o = first_free_offset_reg<8>(ws.occ, hp, ps, lane, ws.occ_lo, ws.occ_hi);
        else {
            if (lane < (int)padded) ws.hs[lane] = hp;
            __syncwarp();
            o = first_free_offset(ws.occ, ws.hs, s, ps, lane, ws.occ_lo, ws.occ_hi);
            __syncwarp();
        }
        if (o == kNone) continue;
        uint32_t q = hk + o;
        q = q >= ps ? q - ps : q;
        mark_if(ws.occ, q, ps, mine && PHB_CHECK(!mine || q < ps));
        __syncwarp();
        *pilot = o + ps * k;
        return PHOBIC_OK;
    }
    return PHOBIC_ERR_SEARCH_LIMIT;
}

// One bucket of more than 32 keys (a few per partition); its keys are read from
// the bucket-ordered copy in global memory, slots go to ws.hs.
__device__ __forceinline__ uint32_t place_large(const WarpSmem &ws, const uint2 *src, uint32_t s, uint32_t ps,
                                                FastMod fm, uint32_t k_lim, int lane, uint32_t *pilot) {
    const uint32_t padded = (s + 3) & ~3u;
    for (uint32_t k = 0; k < k_lim; k++) {
        if (k == kDupCheckAt) {
            bool d = false;
            for (uint32_t t = 0; t + 1 < s; t++) {
                uint2 kt = src[t];
                for (uint32_t i = lane; i < s; i += 32) d |= i > t && src[i].x == kt.x && src[i].y == kt.y;
            }
            if (__any_sync(kFullMask, d)) return PHOBIC_ERR_DUPLICATE_KEY;
        }
        // Hash chunk by chunk; stop at the first chunk that repeats a slot.
        bool dup = false;
        uint32_t done = 0;  // keys hashed (and marked in the collision scratch)
        for (uint32_t c0 = 0; c0 < s && !dup; c0 += 32) {
            const uint32_t i = c0 + lane;
            bool d = false;
            if (i < s) {
                const uint2 key = src[i];
                const uint32_t h = fm.mod(pilot_hash(key.x, key.y, k));
                ws.hs[i] = pack_slot(h);
                const uint32_t bit = 1u << (h & 31);
                d = PHB_CHECK(h < ps) && (atomicOr(&ws.scr[h >> 5], bit) & bit) != 0;
            }
            dup = __any_sync(kFullMask, d);
            done = c0 + 32;
        }
        for (uint32_t i = lane; i < s && i < done; i += 32) ws.scr[unpack_slot(ws.hs[i]) >> 5] = 0;
        __syncwarp();
        if (dup) continue;
        if (s + lane < padded) ws.hs[s + lane] = ws.hs[0];
        __syncwarp();
        const uint32_t o = first_free_offset(ws.occ, ws.hs, s, ps, lane, ws.occ_lo, ws.occ_hi);
        __syncwarp();
        if (o == kNone) continue;
        for (uint32_t i = lane; i < s; i += 32) {
            uint32_t q = unpack_slot(ws.hs[i]) + o;
            q = q >= ps ? q - ps : q;
            if (PHB_CHECK(q < ps)) mark(ws.occ, q, ps);
        }
        __syncwarp();
        *pilot = o + ps * k;
        return PHOBIC_OK;
    }
    return PHOBIC_ERR_SEARCH_LIMIT;
}

// place_large with the bucket's keys in registers: key i = 32 c + lane in key[c],
// loaded once per bucket (C chunks of 32, 32 C >= s).  Each try hashes chunk by
// chunk and stops at the first chunk that repeats a slot, so a bucket that
// collides (the large ones of a partition collide often) hashes about half its
// keys per rejected counter.  Slots go to ws.hs for the offset search and the
// marking, as in place_large.
template <int C>
__device__ __forceinline__ uint32_t place_large_reg(const WarpSmem &ws, const uint2 *src, uint32_t s, uint32_t ps,
                                                    FastMod fm, uint32_t k_lim, int lane, uint32_t *pilot) {
    const uint32_t padded = (s + 3) & ~3u;
    uint2 key[C];
#pragma unroll
    for (int c = 0; c < C; c++) key[c] = 32 * c + lane < (int)s ? src[32 * c + lane] : make_uint2(0, 0);
    for (uint32_t k = 0; k < k_lim; k++) {
        if (k == kDupCheckAt) {
            bool d = false;
            for (uint32_t t = 0; t + 1 < s; t++) {
                uint2 kt = src[t];
#pragma unroll
                for (int c = 0; c < C; c++) {
                    const uint32_t i = 32 * c + lane;
                    d |= i > t && i < s && key[c].x == kt.x && key[c].y == kt.y;
                }
            }
            if (__any_sync(kFullMask, d)) return PHOBIC_ERR_DUPLICATE_KEY;
        }
        bool dup = false;
        int done = 0;  // chunks hashed (and marked in the collision scratch)
#pragma unroll
        for (int c = 0; c < C; c++) {
            if (!dup && 32 * c < (int)s) {
                const uint32_t i = 32 * c + lane;
                bool d = false;
                if (i < s) {
                    const uint32_t h = fm.mod(pilot_hash(key[c].x, key[c].y, k));
                    ws.hs[i] = pack_slot(h);
                    const uint32_t bit = 1u << (h & 31);
                    d = PHB_CHECK(h < ps) && (atomicOr(&ws.scr[h >> 5], bit) & bit) != 0;
                }
                dup = __any_sync(kFullMask, d);
                done = c + 1;
            }
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const uint32_t i = 32 * c + lane;
            if (c < done && i < s) ws.scr[unpack_slot(ws.hs[i]) >> 5] = 0;
        }
        __syncwarp();
        if (dup) continue;
        if (s + lane < padded) ws.hs[s + lane] = ws.hs[0];
        __syncwarp();
        const uint32_t o = first_free_offset(ws.occ, ws.hs, s, ps, lane, ws.occ_lo, ws.occ_hi);
        __syncwarp();
        if (o == kNone) continue;
#pragma unroll
        for (int c = 0; c < C; c++) {
            const uint32_t i = 32 * c + lane;
            if (i < s) {
                uint32_t q = unpack_slot(ws.hs[i]) + o;
                q = q >= ps ? q - ps : q;
                if (PHB_CHECK(q < ps)) mark(ws.occ, q, ps);
            }
        }
        __syncwarp();
        *pilot = o + ps * k;
        return PHOBIC_OK;
    }
    return PHOBIC_ERR_SEARCH_LIMIT;
}

// The bucket-ordered copy of a partition's keys is scratch that lives from the preparation
// to the end of the partition's search.  It is stored with an L2 evict-last policy, so it is
// still in L2 when the search reads it back, while the inputs that are read once (the lower
// hash words and the second read of the bucket ids) are loaded as streaming; once the
// partition is done its 128-byte lines that no other partition shares are discarded from L2
// without being written back.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void st_evict_last(uint2 *p, uint2 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.u32 [%0], {%1, %2}, %3;" ::"l"(p), "r"(v.x), "r"(v.y), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void discard_partition_copy(const uint2 *so, uint32_t ps, int lane) {
    const uintptr_t a = ((uintptr_t)so + 127) & ~(uintptr_t)127;
    const uintptr_t e = ((uintptr_t)(so + ps)) & ~(uintptr_t)127;
    for (uintptr_t x = a + 128u * (uint32_t)lane; x < e; x += 32u * 128u)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(x) : "memory");
}

// Preparation of one partition by one warp: bucket histogram, search order (in
// ws.sched), bucket-ordered keys (in a.sorted), pilot 0 for empty buckets, a clear
// bitmap and collision scratch.  *nonempty = buckets to search; *skip = true when the
// partition is not searched here (reported by the size check).  Returns a status.
__device__ __forceinline__ uint32_t prep_partition(const SearchArgs &a, const WarpSmem &ws, const SetDesc &d,
                                                   uint32_t g, uint32_t p, int lane, uint32_t *nonempty_out,
                                                   bool *skip) {
    *skip = true;
    const uint32_t B = a.buckets;
    const uint32_t base = a.G[(size_t)g * a.gstride];
    const uint32_t end = a.G[(size_t)(g + 1) * a.gstride];
    // K3 placed exactly the keys K1 counted, unless the keys changed in between (loaded
    // with the offsets, so the check adds no wait).
    const uint32_t placed = a.placed ? a.placed[g] : end;
    const uint32_t ps = end - base;
    if (ps > a.cap) return PHOBIC_OK;  // reported by the size check
    if (!PHB_CHECK(base + ps <= a.G[(size_t)a.M * a.gstride])) return PHOBIC_OK;
    *skip = false;
    if (placed != end) return PHOBIC_ERR_KEYS_CHANGED;
    const uint32_t ow = bitmap_words(a.cap);
    uint32_t *pil = d.pilots + p;
    const size_t pstride = d.partitions;

    for (uint32_t i = lane; i < half_words(B); i += 32) ws.cnt32[i] = 0;
    for (uint32_t i = lane; i < ow; i += 32) ws.occ[i] = 0;
    for (uint32_t i = lane; i < 256; i += 32) ws.binPos[i] = 0;  // binPos and binKey
    __syncwarp();

    // Bucket sizes of this partition (bucket_sizes.comp:21-35).
    const uint16_t *bk = a.bkt + base;
#pragma unroll 4
    for (uint32_t i = lane; i < ps; i += 32) {
        // Ids >= B never come from K3 for keys that K1 counted; the clamp keeps a stale
        // record (keys changed during the build) inside the tables.
        const uint32_t b = min((uint32_t)bk[i], B - 1);
        if (PHB_CHECK(b == bk[i])) half_add(ws.cnt32, b);
    }
    __syncwarp();

    // Size histogram in bins 256 - size (sort_sum.comp:56-58,166-170); empty buckets get pilot 0.
    bool over = false;
    for (uint32_t b = lane; b < B; b += 32) {
        uint32_t s = half_get(ws.cnt32, b);
        if (a.debug_sizes) a.debug_sizes[(size_t)g * B + b] = s;
        if (s > kMaxBucket) over = true;
        else if (s && PHB_CHECK(s <= kBins)) half_add(ws.binPos, kBins - s);
        else pil[(size_t)b * pstride] = 0;
    }
    if (__any_sync(kFullMask, over)) return PHOBIC_ERR_BUCKET_OVERFLOW;
    __syncwarp();

    // Exclusive prefix over bins of bucket counts and key counts (sort_sum.comp:184-215);
    // lane L owns bins 8L .. 8L+7, i.e. packed words 4L .. 4L+3 of each table.
    uint32_t c[8], loc = 0, lock = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        uint32_t bin = 8 * lane + j;
        c[j] = half_get(ws.binPos, bin);
        loc += c[j];
        lock += c[j] * (kBins - bin);
    }
    const uint32_t inc = warp_incl_scan(loc, lane), inck = warp_incl_scan(lock, lane);
    const uint32_t nonempty = __shfl_sync(kFullMask, inc, 31);
    uint32_t ex = inc - loc, exk = inck - lock;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
        uint32_t bin = 8 * lane + j;
        const uint32_t ex1 = ex + c[j], exk1 = exk + c[j] * (kBins - bin);
        ws.binPos[bin >> 1] = ex | (ex1 << 16);
        ws.binKey[bin >> 1] = exk | (exk1 << 16);
        ex = ex1 + c[j + 1];
        exk = exk1 + c[j + 1] * (kBins - bin - 1);
    }
    __syncwarp();

    // Search order: within a bin, the higher bucket index first (sort_sum.comp:156).
    uint16_t *cur16 = reinterpret_cast<uint16_t *>(ws.cur32);
    for (uint32_t c0 = 0; c0 < B; c0 += 32) {
        const int bi = (int)B - 1 - (int)(c0 + lane);
        const uint32_t s = bi >= 0 ? half_get(ws.cnt32, bi) : 0u;
        const uint32_t peers = __match_any_sync(kFullMask, s ? s : 0x10000u + lane);
        const uint32_t r = __popc(peers & lanemask_lt());
        const uint32_t bin = kBins - s;
        if (s) {
            const uint32_t j = half_get(ws.binPos, bin) + r, st = half_get(ws.binKey, bin) + r * s;
            if (PHB_CHECK(j < B && st + s <= ps)) {
                ws.sched[j] = st | ((uint32_t)bi << 16);
                cur16[bi] = (uint16_t)st;
            }
        }
        __syncwarp();
        if (s && lane == __ffs(peers) - 1) {
            half_add_n(ws.binPos, bin, __popc(peers));
            half_add_n(ws.binKey, bin, __popc(peers) * s);
        }
        __syncwarp();
    }

    // Keys into bucket order (redistribute_keys.comp:21-53, inside the partition).
    const uint2 *lo = a.lowers + base;
    uint2 *so = a.sorted + base;
    const uint64_t keep = l2_evict_last_policy();
#pragma unroll 4
    for (uint32_t i = lane; i < ps; i += 32) {
        const uint16_t bi = __ldcs(bk + i);
        const uint32_t b = min((uint32_t)bi, B - 1);
        if (!PHB_CHECK(b == bi)) continue;
        const uint32_t pos = half_add(ws.cur32, b);
        if (PHB_CHECK(pos < ps)) st_evict_last(so + pos, __ldcs(lo + i), keep);
    }
    __threadfence_block();
    __syncwarp();
    // The search-phase half of the union: large buckets expect a clear collision scratch.
    for (uint32_t i = lane; i < scr_words(a.cap); i += 32) ws.scr[i] = 0;
    __syncwarp();
    *nonempty_out = nonempty;
    return PHOBIC_OK;
}

// One partition: bucket histogram, search order, bucket-sorted keys, pilots.
__device__ __forceinline__ uint32_t search_partition(const SearchArgs &a, const WarpSmem &ws, const SetDesc &d,
                                                     uint32_t g, uint32_t p, int lane) {
    uint32_t nonempty = 0;
    bool skip = true;
    const uint32_t pst = prep_partition(a, ws, d, g, p, lane, &nonempty, &skip);
    if (skip || pst != PHOBIC_OK) return pst;
    const uint32_t B = a.buckets;
    const uint32_t base = a.G[(size_t)g * a.gstride];
    const uint32_t ps = a.G[(size_t)(g + 1) * a.gstride] - base;
    uint32_t *pil = d.pilots + p;
    const size_t pstride = d.partitions;
    const uint2 *so = a.sorted + base;

    // Pilot search (search.comp:126-175), next bucket's keys prefetched.
    const FastMod fm = FastMod::make(ps ? ps : 1);
    const uint32_t rounds = (ps + 1023) / 1024;
    uint32_t k_lim = 0x80000000u / (ps ? ps : 1);
    if (k_lim > a.k_max) k_lim = a.k_max;
    uint32_t sc_next = nonempty ? ws.sched[0] : 0u;
    uint32_t s_next = nonempty ? half_get(ws.cnt32, sc_next >> 16) : 0u;
    uint2 L_next = lane < (int)s_next ? so[(sc_next & 0xFFFFu) + lane] : make_uint2(0, 0);
    for (uint32_t j = 0; j < nonempty; j++) {
        const uint32_t sc = sc_next, s = s_next;
        const uint2 L = L_next;
        const uint32_t b = sc >> 16, st = sc & 0xFFFFu;
        if (j + 1 < nonempty) {
            sc_next = ws.sched[j + 1];
            s_next = half_get(ws.cnt32, sc_next >> 16);
            L_next = lane < (int)s_next ? so[(sc_next & 0xFFFFu) + lane] : make_uint2(0, 0);
        }
        uint32_t pilot = 0;
        const uint32_t st_code = s <= 4 && rounds <= 3 ? place_batched<4>(ws, L, s, ps, fm, k_lim, rounds, lane, &pilot)
                                 : s <= 8 && rounds <= 3 ? place_batched<8>(ws, L, s, ps, fm, k_lim, rounds, lane, &pilot)
                                 : s <= 32 ? place_small(ws, L, s, ps, fm, k_lim, rounds, lane, &pilot)
                                 : s <= 64  ? place_large_reg<2>(ws, so + st, s, ps, fm, k_lim, lane, &pilot)
                                            : place_large(ws, so + st, s, ps, fm, k_lim, lane, &pilot);
        if (st_code != PHOBIC_OK) return st_code;
        if (lane == 0 && PHB_CHECK(b < B)) pil[(size_t)b * pstride] = pilot;
    }
    __syncwarp();
    discard_partition_copy(so, ps, lane);
    return PHOBIC_OK;
}

// ------------------------------------------------------------------ k-split groups
//
// For builds with far fewer partitions than warp slots (small key sets, where one
// warp per partition leaves most of the GPU idle and each partition's search is
// bound by the latency of its sequential tries), a group of W warps searches one
// partition: in each step, warp w tries pilot counter k0 + w for the current bucket
// (hash, collision test, offset scan over all of [0, ps)).  The step's outcomes are
// exchanged in shared memory and read in k order, so the bucket takes the smallest k
// that has a free offset, with that k's smallest offset: the result of trying
// k = 0, 1, 2, ... one at a time (search.comp:105-124).  Every warp then marks the
// winning slots itself (the marks are idempotent), so no warp reads the bitmap before
// its own copy of the marks is in place.
constexpr uint32_t kTryNone = 0, kTryFound = 1, kTryDup = 2, kTryLimit = 3;

__device__ __forceinline__ void group_bar(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Per-warp scratch of warps 1..W-1 of a group (warp 0 uses the union of carve()).
__host__ __device__ __forceinline__ size_t group_extra_words(uint32_t cap) {
    return ((size_t)kHsWords + scr_words(cap) + 3) & ~size_t(3);
}
// Exchange words: [2 parities][W] outcomes, the control words (job, nonempty, committed,
// status), and the bucket pipeline's results: [W] (code << 24 | k, offset) pairs and [W][32]
// slots (padded).
__host__ __device__ __forceinline__ size_t group_xch_words(int W) {
    return ((size_t)2 * W + 4 + 2 * (size_t)W + 32 * (size_t)W + 3) & ~size_t(3);
}
__host__ __device__ __forceinline__ size_t group_words(uint32_t B, uint32_t cap, int W) {
    return warp_words(B, cap) + (size_t)(W - 1) * group_extra_words(cap) + group_xch_words(W);
}

// One try of a pilot counter for a bucket of s <= 32 keys, hk holding key `lane`'s slot
// under that counter: the collision test and offset scan of place_small.  kTryFound with
// *o, else kTryNone.
__device__ __forceinline__ uint32_t try_small(const WarpSmem &ws, uint32_t s, uint32_t ps, uint32_t hk,
                                              uint32_t rounds, int lane, uint32_t *o_out) {
    const bool mine = lane < (int)s;
    const uint32_t padded = (s + 3) & ~3u;
    const uint32_t h = mine ? hk : (0x80000000u | lane);
    if (s > 1) {
        uint32_t m = __match_any_sync(kFullMask, h);
        if (__any_sync(kFullMask, mine && (m & (m - 1)) != 0)) return kTryNone;
    }
    const uint32_t hp = pack_slot(__shfl_sync(kFullMask, h, mine ? lane : 0));
    uint32_t o;
    if (s <= 8 && rounds <= 3) {
        if (s <= 4) o = first_free_offset_unr<4>(ws.occ, hp, ps, rounds, lane, ws.occ_lo, ws.occ_hi);
        else o = first_free_offset_unr<8>(ws.occ, hp, ps, rounds, lane, ws.occ_lo, ws.occ_hi);
    } else if (s <= 4) o = first_free_offset_reg<4>(ws.occ, hp, ps, lane, ws.occ_lo, ws.occ_hi);
    else if (s <= 8) o = first_free_offset_reg<8>(ws.occ, hp, ps, lane, ws.occ_lo, ws.occ_hi);
    else {
        if (lane < (int)padded) ws.hs[lane] = hp;
        __syncwarp();
        o = first_free_offset(ws.occ, ws.hs, s, ps, lane, ws.occ_lo, ws.occ_hi);
        __syncwarp();
    }
    if (o == kNone) return kTryNone;
    *o_out = o;
    return kTryFound;
}

// One try of pilot counter k for a bucket of more than 32 keys read from src: the
// chunked collision test and offset scan of place_large.
__device__ __forceinline__ uint32_t try_large(const WarpSmem &ws, const uint2 *src, uint32_t s, uint32_t ps,
                                              FastMod fm, uint32_t k, int lane, uint32_t *o_out) {
    const uint32_t padded = (s + 3) & ~3u;
    bool dup = false;
    uint32_t done = 0;
    for (uint32_t c0 = 0; c0 < s && !dup; c0 += 32) {
        const uint32_t i = c0 + lane;
        bool d = false;
        if (i < s) {
            const uint2 key = src[i];
            const uint32_t h = fm.mod(pilot_hash(key.x, key.y, k));
            ws.hs[i] = pack_slot(h);
            const uint32_t bit = 1u << (h & 31);
            d = PHB_CHECK(h < ps) && (atomicOr(&ws.scr[h >> 5], bit) & bit) != 0;
        }
        dup = __any_sync(kFullMask, d);
        done = c0 + 32;
    }
    for (uint32_t i = lane; i < s && i < done; i += 32) ws.scr[unpack_slot(ws.hs[i]) >> 5] = 0;
    __syncwarp();
    if (dup) return kTryNone;
    if (s + lane < padded) ws.hs[s + lane] = ws.hs[0];
    __syncwarp();
    const uint32_t o = first_free_offset(ws.occ, ws.hs, s, ps, lane, ws.occ_lo, ws.occ_hi);
    __syncwarp();
    if (o == kNone) return kTryNone;
    *o_out = o;
    return kTryFound;
}

// Whether two of the s keys read from src are identical (the check at pilot counter
// kDupCheckAt of place_large).
__device__ __noinline__ bool has_duplicate_key_src(const uint2 *src, uint32_t s, int lane) {
    bool d = false;
    for (uint32_t t = 0; t + 1 < s; t++) {
        const uint2 kt = src[t];
        for (uint32_t i = lane; i < s; i += 32) d |= i > t && src[i].x == kt.x && src[i].y == kt.y;
    }
    return __any_sync(kFullMask, d);
}

// Marks the slots (h_i + o) mod ps of the bucket's keys at pilot counter k.
__device__ __forceinline__ void mark_bucket(const WarpSmem &ws, uint2 L, const uint2 *src, uint32_t s, uint32_t ps,
                                            FastMod fm, uint32_t k, uint32_t o, int lane) {
    if (s <= 32) {
        if (lane < (int)s) {
            uint32_t q = fm.mod(pilot_hash(L.x, L.y, k)) + o;
            q = q >= ps ? q - ps : q;
            if (PHB_CHECK(q < ps)) mark(ws.occ, q, ps);
        }
    } else {
        for (uint32_t i = lane; i < s; i += 32) {
            const uint2 key = src[i];
            uint32_t q = fm.mod(pilot_hash(key.x, key.y, k)) + o;
            q = q >= ps ? q - ps : q;
            if (PHB_CHECK(q < ps)) mark(ws.occ, q, ps);
        }
    }
    __syncwarp();
}

// Group kernel: kSearchWarps / W groups per CTA, each a persistent searcher over the
// partition queue.  Warp 0 of a group prepares the partition (prep_partition); all W
// warps then search its buckets in k-split steps.
// Small builds leave most SMs idle, so the group kernel is not held to the one-warp
// kernel's 4 CTAs per SM (64 registers): 2 CTAs per SM keep it free of spills.
// Bucket pipeline (PIPE): for buckets of at most 32 keys (the tail of the search order),
// warp w searches bucket j + w completely (smallest k, then smallest o) on the bitmap as it
// stands, without marking.  Warp 0 then commits the W results in order: a result is kept
// while its slots are still free after the results before it were marked.  That keeps the
// sequential answer: the bitmap only gains occupied slots, so a (k, o) valid on the later
// state was valid on the earlier one, and the smallest valid pair on the earlier state, if
// still valid, is the smallest on the later one.  A pilot limit or duplicate keys found on the
// earlier state hold on the later one too.  The first result that conflicts is searched again
// in the next step.
template <int W, bool PIPE>
__global__ void __launch_bounds__(kSearchWarps * 32, 2) k_search_group(SearchArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = warp / W, w = warp % W;
    const uint32_t bar_id = 1 + grp, bar_n = 32 * W;
    uint32_t *gbase = smem + (size_t)grp * group_words(a.buckets, a.cap, W);
    WarpSmem ws = carve(gbase, a.buckets, a.cap);
    if (w > 0) {
        ws.hs = gbase + warp_words(a.buckets, a.cap) + (size_t)(w - 1) * group_extra_words(a.cap);
        ws.scr = ws.hs + kHsWords;
    }
    uint32_t *xch = gbase + warp_words(a.buckets, a.cap) + (size_t)(W - 1) * group_extra_words(a.cap);
    uint32_t *ctl = xch + 2 * W;  // [0] job, [1] nonempty, [2] committed, [3] status
    uint32_t *pres = ctl + 4;     // [W] pairs: code << 24 | k, offset
    uint32_t *pslots = pres + 2 * W;  // [W][32] slots of each warp's result
    uint32_t par = 0;
    for (;;) {
        if (w == 0 && lane == 0) ctl[0] = atomicAdd(a.queue, 1u);
        group_bar(bar_id, bar_n);
        const uint32_t g = ctl[0];
        if (g >= a.M) break;
        const uint32_t s_idx = a.nsets == 1 ? 0u : find_set(a.part_base, a.nsets, g);
        const SetDesc &d = a.sets[s_idx];
        const uint32_t p = g - d.part_base;
        // Warp 0 prepares; ctl[1] = nonempty buckets, or 0xFFFFFFFF when there is nothing to search.
        if (w == 0) {
            uint32_t ctl1 = 0xFFFFFFFFu;
            if (!fatal_before_search(*reinterpret_cast<volatile unsigned long long *>(&a.err[s_idx]))) {
                if (lane == 0 && d.part_off) {
                    const uint32_t g0 = a.G[(size_t)d.part_base * a.gstride];
                    d.part_off[p] = a.G[(size_t)g * a.gstride] - g0;
                    if (p + 1 == d.partitions) d.part_off[p + 1] = a.G[(size_t)(g + 1) * a.gstride] - g0;
                }
                uint32_t nonempty = 0;
                bool skip = true;
                const uint32_t code = prep_partition(a, ws, d, g, p, lane, &nonempty, &skip);
                if (code != PHOBIC_OK && lane == 0) report_error(&a.err[s_idx], p, code);
                if (!skip && code == PHOBIC_OK) ctl1 = nonempty;
            }
            if (lane == 0) ctl[1] = ctl1;
        } else {
            for (uint32_t i = lane; i < scr_words(a.cap); i += 32) ws.scr[i] = 0;
        }
        group_bar(bar_id, bar_n);
        const uint32_t nonempty = ctl[1];
        if (nonempty != 0xFFFFFFFFu) {
            const uint32_t base = a.G[(size_t)g * a.gstride];
            const uint32_t ps = a.G[(size_t)(g + 1) * a.gstride] - base;
            const uint2 *so = a.sorted + base;
            uint32_t *pil = d.pilots + p;
            const size_t pstride = d.partitions;
            const FastMod fm = FastMod::make(ps ? ps : 1);
            const uint32_t rounds = (ps + 1023) / 1024;
            uint32_t k_lim = 0x80000000u / (ps ? ps : 1);
            if (k_lim > a.k_max) k_lim = a.k_max;
            uint32_t err = PHOBIC_OK;
            for (uint32_t j = 0; j < nonempty && err == PHOBIC_OK; j++) {
                const uint32_t sc = ws.sched[j];
                const uint32_t b = sc >> 16, st = sc & 0xFFFFu;
                const uint32_t s = half_get(ws.cnt32, b);
                const uint2 *src = so + st;
                if (PIPE && s <= 32) {  // every later bucket is as small (search order: size descending)
                    const uint32_t jw = j + w;
                    if (jw < nonempty) {
                        const uint32_t scw = ws.sched[jw];
                        const uint32_t sw = half_get(ws.cnt32, scw >> 16);
                        const uint2 Lw = lane < (int)sw ? so[(scw & 0xFFFFu) + lane] : make_uint2(0, 0);
                        uint32_t code = kTryLimit, kk = 0, o = 0;
                        if (sw <= 8 && rounds <= 3) {  // several counters hashed at once
                            uint32_t q = 0;
                            const uint32_t st = sw <= 4 ? place_batched<4, false>(ws, Lw, sw, ps, fm, k_lim, rounds,
                                                                                  lane, nullptr, &kk, &o, &q)
                                                        : place_batched<8, false>(ws, Lw, sw, ps, fm, k_lim, rounds,
                                                                                  lane, nullptr, &kk, &o, &q);
                            code = st == PHOBIC_OK                  ? kTryFound
                                   : st == PHOBIC_ERR_DUPLICATE_KEY ? kTryDup
                                                                    : kTryLimit;
                            if (code == kTryFound && lane < (int)sw) pslots[32 * w + lane] = q;
                        } else {
                            // The hash of counter k + 1 is formed while counter k is tested.
                            uint32_t hk_next = fm.mod(pilot_hash(Lw.x, Lw.y, 0u)), hk = 0;
                            for (uint32_t k = 0; k < k_lim; k++) {
                                if (k == kDupCheckAt && sw > 1 && has_duplicate_key(Lw, sw, lane)) {
                                    code = kTryDup;
                                    break;
                                }
                                hk = hk_next;
                                hk_next = fm.mod(pilot_hash(Lw.x, Lw.y, k + 1));
                                if (try_small(ws, sw, ps, hk, rounds, lane, &o) == kTryFound) {
                                    code = kTryFound;
                                    kk = k;
                                    break;
                                }
                            }
                            if (code == kTryFound && lane < (int)sw) {
                                const uint32_t q = hk + o;
                                pslots[32 * w + lane] = q >= ps ? q - ps : q;
                            }
                        }
                        if (lane == 0) {
                            pres[2 * w] = (code << 24) | (kk & 0xFFFFFFu);
                            pres[2 * w + 1] = o;
                        }
                    }
                    group_bar(bar_id, bar_n);
                    if (w == 0) {
                        uint32_t committed = 0, e = PHOBIC_OK;
                        for (uint32_t v = 0; v < (uint32_t)W && j + v < nonempty; v++) {
                            const uint32_t r0 = pres[2 * v], rcode = r0 >> 24;
                            if (rcode != kTryFound) {
                                e = rcode == kTryDup ? PHOBIC_ERR_DUPLICATE_KEY : PHOBIC_ERR_SEARCH_LIMIT;
                                break;
                            }
                            const uint32_t scv = ws.sched[j + v], bv = scv >> 16;
                            const uint32_t sv = half_get(ws.cnt32, bv);
                            const bool mine = lane < (int)sv;
                            const uint32_t q = mine ? pslots[32 * v + lane] : 0u;
                            const bool taken = mine && PHB_CHECK(q < ps) && ((ws.occ[q >> 5] >> (q & 31)) & 1u);
                            if (__any_sync(kFullMask, taken)) break;  // searched again in the next step
                            mark_if(ws.occ, q, ps, mine && PHB_CHECK(!mine || q < ps));
                            __syncwarp();
                            if (lane == 0 && PHB_CHECK(bv < a.buckets))
                                pil[(size_t)bv * pstride] = pres[2 * v + 1] + ps * (r0 & 0xFFFFFFu);
                            committed++;
                        }
                        if (lane == 0) {
                            ctl[2] = committed;
                            ctl[3] = e;
                        }
                    }
                    group_bar(bar_id, bar_n);
                    err = ctl[3];
                    j += ctl[2];
                    j--;  // the loop's increment
                    continue;
                }
                const uint2 L = lane < (int)s && s <= 32 ? src[lane] : make_uint2(0, 0);
                for (uint32_t k0 = 0;; k0 += W) {
                    const uint32_t k = k0 + w;
                    uint32_t code = kTryNone, o = 0;
                    if (k >= k_lim) code = kTryLimit;
                    else if (k == kDupCheckAt && s > 1 &&
                             (s <= 32 ? has_duplicate_key(L, s, lane) : has_duplicate_key_src(src, s, lane)))
                        code = kTryDup;
                    else code = s <= 32 ? try_small(ws, s, ps, fm.mod(pilot_hash(L.x, L.y, k)), rounds, lane, &o)
                                        : try_large(ws, src, s, ps, fm, k, lane, &o);
                    if (lane == 0) xch[par * W + w] = (code << 16) | (o & 0xFFFFu);
                    group_bar(bar_id, bar_n);
                    uint32_t win = kTryNone << 16, v = 0;
                    for (; v < (uint32_t)W; v++) {
                        win = xch[par * W + v];
                        if ((win >> 16) != kTryNone) break;
                    }
                    par ^= 1u;
                    const uint32_t wcode = win >> 16;
                    if (wcode == kTryNone) continue;
                    if (wcode == kTryFound) {
                        const uint32_t kw = k0 + v, ow = win & 0xFFFFu;
                        mark_bucket(ws, L, src, s, ps, fm, kw, ow, lane);
                        if (w == 0 && lane == 0 && PHB_CHECK(b < a.buckets)) pil[(size_t)b * pstride] = ow + ps * kw;
                    } else {
                        err = wcode == kTryDup ? PHOBIC_ERR_DUPLICATE_KEY : PHOBIC_ERR_SEARCH_LIMIT;
                    }
                    break;
                }
            }
            if (err != PHOBIC_OK && w == 0 && lane == 0) report_error(&a.err[s_idx], p, err);
        }
        // Everyone is done with this partition's tables before warp 0 fetches and prepares the next.
        group_bar(bar_id, bar_n);
        if (w == 0 && nonempty != 0xFFFFFFFFu) {
            const uint32_t base = a.G[(size_t)g * a.gstride];
            discard_partition_copy(a.sorted + base, a.G[(size_t)(g + 1) * a.gstride] - base, lane);
        }
    }
}

}  // namespace

unsigned int check_line_search(bool reset) { return read_check_line(reset); }

size_t search_warp_smem(uint32_t buckets, uint32_t cap) { return 4 * warp_words(buckets, cap); }

int search_warps_per_cta(uint32_t buckets, uint32_t cap) {
    if (cap > 65535 || buckets > 65535) return 0;
    size_t fit = kSearchSmemLimit / search_warp_smem(buckets, cap);
    return (int)(fit < (size_t)kSearchWarps ? fit : (size_t)kSearchWarps);
}

__global__ void __launch_bounds__(kSearchWarps * 32, kSearchCtasPerSm) k_search(SearchArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const WarpSmem ws = carve(smem + (size_t)warp * warp_words(a.buckets, a.cap), a.buckets, a.cap);
    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(a.queue, 1u);
        g = __shfl_sync(kFullMask, g, 0);
        if (g >= a.M) break;
        const uint32_t s = a.nsets == 1 ? 0u : find_set(a.part_base, a.nsets, g);
        if (fatal_before_search(*reinterpret_cast<volatile unsigned long long *>(&a.err[s]))) continue;
        const SetDesc &d = a.sets[s];
        const uint32_t p = g - d.part_base;
        if (lane == 0 && d.part_off) {
            const uint32_t g0 = a.G[(size_t)d.part_base * a.gstride];
            d.part_off[p] = a.G[(size_t)g * a.gstride] - g0;
            if (p + 1 == d.partitions) d.part_off[p + 1] = a.G[(size_t)(g + 1) * a.gstride] - g0;
        }
        const uint32_t code = search_partition(a, ws, d, g, p, lane);
        if (code != PHOBIC_OK && lane == 0) report_error(&a.err[s], p, code);
    }
}

size_t search_group_smem(uint32_t buckets, uint32_t cap, int W) { return 4 * group_words(buckets, cap, W); }

template <int W, bool PIPE>
static cudaError_t launch_group(const SearchArgs &a, int sm_count, cudaStream_t st) {
    constexpr int groups = kSearchWarps / W;
    const size_t smem = (size_t)groups * search_group_smem(a.buckets, a.cap, W);
    if (smem > kSearchSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = allow_dynamic_smem(k_search_group<W, PIPE>, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search_group<W, PIPE>, kSearchWarps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const uint64_t want = (a.M + groups - 1) / groups;
    const int grid = (int)std::min<uint64_t>(want, (uint64_t)per_sm * sm_count);
    k_search_group<W, PIPE><<<grid, kSearchWarps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

SearchShape search_shape_for(uint32_t partitions, int sm_count) {
    // Measured on a B200 (the autotuner's ladder, three key sets per size, six parameter
    // sets): bucket pipelines of 8 warps are fastest up to 256 partitions, of 4 warps up to
    // 512, of 2 warps up to 1024; one warp per partition beyond.  A group must fit one wave
    // of the group kernel (2 CTAs of kSearchWarps warps per SM).
    const uint64_t wave = (uint64_t)(sm_count > 0 ? sm_count : 148) * 2 * kSearchWarps;
    SearchShape sh;
    sh.group = 1;
    if ((uint64_t)partitions * 8 <= wave && partitions <= 256) sh = SearchShape{8, true};
    else if ((uint64_t)partitions * 4 <= wave && partitions <= 512) sh = SearchShape{4, true};
    else if ((uint64_t)partitions * 2 <= wave && partitions <= 1024) sh = SearchShape{2, true};
    return sh;
}

cudaError_t launch_search(const SearchArgs &a, int sm_count, cudaStream_t st, SearchShape shape) {
    if (a.M == 0) return cudaSuccess;
    if (shape.group == 0) shape = search_shape_for(a.M, sm_count);
    const int group = shape.group;
    const bool pipeline = shape.pipeline;
    if (group == 2 || group == 4 || group == 8) {
        cudaError_t e;
        if (pipeline)
            e = group == 2 ? launch_group<2, true>(a, sm_count, st)
                : group == 4 ? launch_group<4, true>(a, sm_count, st) : launch_group<8, true>(a, sm_count, st);
        else
            e = group == 2 ? launch_group<2, false>(a, sm_count, st)
                : group == 4 ? launch_group<4, false>(a, sm_count, st) : launch_group<8, false>(a, sm_count, st);
        if (e != cudaErrorInvalidValue) return e;
        cudaGetLastError();  // the group's tables do not fit: one warp per partition
    }
    const int warps = search_warps_per_cta(a.buckets, a.cap);
    if (warps < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)warps * search_warp_smem(a.buckets, a.cap);
    cudaError_t e = allow_dynamic_smem(k_search, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint64_t want = (a.M + warps - 1) / warps;
    int grid = (int)std::min<uint64_t>(want, (uint64_t)per_sm * sm_count);
    k_search<<<grid, warps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace phobicb200
