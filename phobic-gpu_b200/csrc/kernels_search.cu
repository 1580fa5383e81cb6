// K4: per-partition bucket sort and pilot search, one warp per partition.
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
// The offset search tests 32 offsets per lane with one funnel shift per key:
// the occupancy bitmap keeps a copy of its first 32 bits after bit ps, so the
// 32-bit window starting at any slot < ps reads circularly.  A warp covers
// 1024 consecutive offsets per round; the first lane with a free window holds
// the smallest valid offset.
#include "kernels.cuh"

namespace phobicb200 {

namespace {

constexpr int kMaxPerLane = kMaxBucket / 32;  // keys of one bucket held per lane

__device__ __forceinline__ uint32_t occ_words(uint32_t cap) { return (cap + 31) / 32 + 2; }

struct WarpSmem {
    uint32_t *cnt;    // [B] keys per bucket
    uint32_t *cur;    // [B] scatter cursor; after the scatter: bucket end
    uint16_t *order;  // [B] bucket ids in search order
    uint32_t *occ;    // [OW] occupied slots, bits [ps, ps+32) mirror [0, 32)
    uint32_t *scr;    // [OW] scratch bitmap for collision checks of large buckets
    uint32_t *binPos; // [256] bin cursor in `order`      (prep phase)
    uint32_t *binKey; // [256] bin cursor in key positions (prep phase)
    uint32_t *hs;     // [256] slots of the current bucket (search phase, aliases binPos)
};

__host__ __device__ __forceinline__ size_t warp_words(uint32_t B, uint32_t cap) {
    return 2 * (size_t)B + (B + 1) / 2 + 2 * (size_t)((cap + 31) / 32 + 2) + 512;
}

__device__ __forceinline__ WarpSmem carve(uint32_t *base, uint32_t B, uint32_t cap) {
    WarpSmem w;
    uint32_t ow = occ_words(cap);
    w.cnt = base;
    w.cur = w.cnt + B;
    w.order = reinterpret_cast<uint16_t *>(w.cur + B);
    w.occ = w.cur + B + (B + 1) / 2;
    w.scr = w.occ + ow;
    w.binPos = w.scr + ow;
    w.binKey = w.binPos + 256;
    w.hs = w.binPos;
    return w;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(kFullMask, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

}  // namespace

size_t search_warp_smem(uint32_t buckets, uint32_t cap) { return 4 * warp_words(buckets, cap); }

__global__ void __launch_bounds__(kSearchWarps * 32) k_search(SearchArgs a) {
    extern __shared__ uint32_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t p = blockIdx.x * (blockDim.x >> 5) + warp;
    if (p >= a.partitions) return;
    if (fatal_before_search(*reinterpret_cast<volatile unsigned long long *>(a.err))) return;

    const uint32_t B = a.buckets;
    WarpSmem ws = carve(smem + (size_t)warp * warp_words(B, a.cap), B, a.cap);
    const uint32_t base = a.part_off[p];
    const uint32_t ps = a.part_off[p + 1] - base;
    if (ps > a.cap) return;  // reported by the scan
    const uint32_t ow = occ_words(a.cap);

    for (uint32_t i = lane; i < B; i += 32) ws.cnt[i] = 0;
    for (uint32_t i = lane; i < ow; i += 32) ws.occ[i] = 0, ws.scr[i] = 0;
    for (uint32_t i = lane; i < 512; i += 32) ws.binPos[i] = 0;
    __syncwarp();

    // Bucket sizes (bucket_sizes.comp:21-35, restricted to this partition).
    for (uint32_t i = lane; i < ps; i += 32) atomicAdd(&ws.cnt[a.bkt[base + i]], 1u);
    __syncwarp();

    // Size histogram in bins 256 - size (sort_sum.comp:56-58,166-170); empty buckets get pilot 0.
    bool over = false;
    for (uint32_t b = lane; b < B; b += 32) {
        uint32_t s = ws.cnt[b];
        if (a.debug_sizes) a.debug_sizes[(size_t)p * B + b] = s;
        if (s > kMaxBucket) over = true;
        else if (s) atomicAdd(&ws.binPos[kBins - s], 1u);
        else a.pilots[(size_t)b * a.partitions + p] = 0;
    }
    if (__any_sync(kFullMask, over)) {
        if (lane == 0) report_error(a.err, p, PHOBIC_ERR_BUCKET_OVERFLOW);
        return;
    }
    __syncwarp();

    // Exclusive prefix over bins of bucket counts and of key counts (sort_sum.comp:184-215).
    uint32_t c[8], loc = 0, lock = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        uint32_t bin = 8 * lane + j;
        c[j] = ws.binPos[bin];
        loc += c[j];
        lock += c[j] * (kBins - bin);
    }
    uint32_t inc = warp_incl_scan(loc, lane), inck = warp_incl_scan(lock, lane);
    const uint32_t nonempty = __shfl_sync(kFullMask, inc, 31);
    uint32_t ex = inc - loc, exk = inck - lock;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; j++) {
        uint32_t bin = 8 * lane + j;
        ws.binPos[bin] = ex;
        ws.binKey[bin] = exk;
        ex += c[j];
        exk += c[j] * (kBins - bin);
    }
    __syncwarp();

    // Search order: within a bin, higher bucket index first (sort_sum.comp:156).
    for (uint32_t c0 = 0; c0 < B; c0 += 32) {
        int bi = (int)B - 1 - (int)(c0 + lane);
        uint32_t s = bi >= 0 ? ws.cnt[bi] : 0u;
        uint32_t peers = __match_any_sync(kFullMask, s ? s : 0x10000u + lane);
        uint32_t r = __popc(peers & lanemask_lt());
        uint32_t bin = kBins - s;
        if (s) {
            ws.order[ws.binPos[bin] + r] = (uint16_t)bi;
            ws.cur[bi] = ws.binKey[bin] + r * s;
        }
        __syncwarp();
        if (s && lane == __ffs(peers) - 1) {
            ws.binPos[bin] += __popc(peers);
            ws.binKey[bin] += __popc(peers) * s;
        }
        __syncwarp();
    }

    // Keys into bucket order (redistribute_keys.comp:21-53, inside the partition).
    for (uint32_t i = lane; i < ps; i += 32) {
        uint32_t b = a.bkt[base + i];
        uint32_t pos = atomicAdd(&ws.cur[b], 1u);
        a.sorted[base + pos] = a.lowers[base + i];
    }
    __threadfence_block();
    __syncwarp();

    const FastMod fm = FastMod::make(ps ? ps : 1);
    uint32_t k_lim = 0x80000000u / (ps ? ps : 1);
    if (k_lim > a.k_max) k_lim = a.k_max;

    for (uint32_t j = 0; j < nonempty; j++) {
        const uint32_t b = ws.order[j];
        const uint32_t s = ws.cnt[b];
        const uint32_t st = ws.cur[b] - s;
        uint2 L[kMaxPerLane];
        uint32_t H[kMaxPerLane];
#pragma unroll
        for (int r = 0; r < kMaxPerLane; r++) {
            uint32_t i = lane + 32 * r;
            L[r] = i < s ? a.sorted[base + st + i] : make_uint2(0, 0);
        }
        bool placed = false;
        for (uint32_t k = 0; k < k_lim; k++) {
            if (k == kDupCheckAt && s > 1) {
                bool dupk = false;
                for (uint32_t t = 0; t < s; t++) {
                    uint2 kt = a.sorted[base + st + t];
#pragma unroll
                    for (int r = 0; r < kMaxPerLane; r++) {
                        uint32_t i = lane + 32 * r;
                        if (i < s && i > t && L[r].x == kt.x && L[r].y == kt.y) dupk = true;
                    }
                }
                if (__any_sync(kFullMask, dupk)) {
                    if (lane == 0) report_error(a.err, p, PHOBIC_ERR_DUPLICATE_KEY);
                    return;
                }
            }
            // Slots for this k (search.comp:44-70).
#pragma unroll
            for (int r = 0; r < kMaxPerLane; r++) {
                uint32_t i = lane + 32 * r;
                if (i < s) {
                    H[r] = fm.mod(pilot_hash(L[r].x, L[r].y, k));
                    ws.hs[i] = H[r];
                }
            }
            bool dup = false;
            if (s > 1) {
                if (s <= 32) {
                    uint32_t key = lane < (int)s ? H[0] : 0x80000000u | lane;
                    uint32_t m = __match_any_sync(kFullMask, key);
                    dup = __any_sync(kFullMask, lane < (int)s && __popc(m) > 1);
                } else {
                    bool d = false;
#pragma unroll
                    for (int r = 0; r < kMaxPerLane; r++) {
                        uint32_t i = lane + 32 * r;
                        if (i < s) {
                            uint32_t bit = 1u << (H[r] & 31);
                            if (atomicOr(&ws.scr[H[r] >> 5], bit) & bit) d = true;
                        }
                    }
                    dup = __any_sync(kFullMask, d);
#pragma unroll
                    for (int r = 0; r < kMaxPerLane; r++) {
                        uint32_t i = lane + 32 * r;
                        if (i < s) ws.scr[H[r] >> 5] = 0;
                    }
                }
            }
            __syncwarp();
            if (dup) continue;

            // Smallest free offset (search.comp:72-103): lane L tests o in [w, w+32).
            uint32_t o = 0xFFFFFFFFu;
            for (uint32_t w0 = 0; w0 < ps; w0 += 1024) {
                const uint32_t w = w0 + 32 * lane;
                const bool live = w < ps;
                const uint32_t wl = live ? w : 0u;
                uint32_t bad = live ? 0u : kFullMask;
                for (uint32_t i = 0; i < s; i++) {
                    uint32_t x = ws.hs[i] + wl;
                    if (x >= ps) x -= ps;
                    uint32_t wi = x >> 5;
                    bad |= __funnelshift_r(ws.occ[wi], ws.occ[wi + 1], x & 31);
                    if ((i & 7) == 7 && __all_sync(kFullMask, bad == kFullMask)) break;
                }
                uint32_t valid = ~bad;
                if (live && ps - w < 32) valid &= (1u << (ps - w)) - 1u;
                uint32_t ball = __ballot_sync(kFullMask, valid != 0);
                if (ball) {
                    int f = __ffs(ball) - 1;
                    uint32_t vf = __shfl_sync(kFullMask, valid, f);
                    o = w0 + 32 * f + __ffs(vf) - 1;
                    break;
                }
            }
            if (o == 0xFFFFFFFFu) continue;

            // Mark the slots (search.comp:113-117) and store the pilot (:122, :170-174).
#pragma unroll
            for (int r = 0; r < kMaxPerLane; r++) {
                uint32_t i = lane + 32 * r;
                if (i < s) {
                    uint32_t q = H[r] + o;
                    if (q >= ps) q -= ps;
                    atomicOr(&ws.occ[q >> 5], 1u << (q & 31));
                    if (q < 32) {
                        uint32_t m = q + ps;
                        atomicOr(&ws.occ[m >> 5], 1u << (m & 31));
                    }
                }
            }
            __syncwarp();
            if (lane == 0) a.pilots[(size_t)b * a.partitions + p] = o + ps * k;
            placed = true;
            break;
        }
        if (!placed) {
            if (lane == 0) report_error(a.err, p, PHOBIC_ERR_SEARCH_LIMIT);
            return;
        }
    }
}

int search_warps_per_cta(uint32_t buckets, uint32_t cap) {
    size_t per_warp = search_warp_smem(buckets, cap);
    size_t fit = kSearchSmemLimit / per_warp;
    return (int)(fit < (size_t)kSearchWarps ? fit : (size_t)kSearchWarps);
}

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.partitions == 0) return cudaSuccess;
    int warps = search_warps_per_cta(a.buckets, a.cap);
    if (warps < 1) return cudaErrorInvalidValue;
    size_t smem = (size_t)warps * search_warp_smem(a.buckets, a.cap);
    cudaError_t e = cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    uint32_t grid = (a.partitions + warps - 1) / warps;
    k_search<<<grid, warps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace phobicb200
