// K3 as a two-pass radix partition: keys -> partition-contiguous records.
//
// Replaces apply_partition_offset.comp:9-18 and redistribute_keys.comp:21-53 up
// to the order inside a partition (K4 sorts a partition by bucket in shared
// memory).  One scattered store per key, as in a single pass with a cursor per
// partition, leaves HBM and L2 doing 8- and 2-byte partial-sector writes; here
// every store is part of a contiguous run:
//
//   pass 1 (k_bin)    a tile of kPartTile keys is hashed, counting-sorted in
//                     shared memory by coarse bin (gp >> wshift, at most kMaxBins
//                     bins of 2^wshift partitions) and written bin by bin to the
//                     record array `inter`, each run at a bin cursor taken with
//                     one global atomic per (tile, bin).
//   pass 2 (k_place)  a tile of `inter` (one or two coarse bins) is
//                     counting-sorted by partition and written run by run to
//                     `lowers` / `bkt`, each run at a partition cursor taken with
//                     one global atomic per (tile, partition).  A tile whose
//                     partitions span more than kLocalRange ids (only for tiny
//                     partitions) places its records one atomic at a time.
//
// The cursors start at the partition offsets of K2 (bin cursor = offset of the
// bin's first partition), so the records of partition g fill exactly
// [G[g], G[g + 1]); their order inside the partition is unspecified, which the
// search does not depend on.
#include "kernels.cuh"

namespace phobicb200 {

namespace {

struct SetCache {
    uint32_t s = 0xFFFFFFFFu;
    uint64_t lo = 0, hi = 0;
    const void *data = nullptr;
    const uint64_t *offsets = nullptr;
    uint32_t part_base = 0, partitions = 0;

    __device__ __forceinline__ void locate(const MapArgs &a, uint64_t g) {
        if (g >= lo && g < hi) return;
        s = a.nsets == 1 ? 0u : find_set(a.key_base, a.nsets, g);
        const SetDesc &d = a.sets[s];
        lo = d.key_base;
        hi = d.key_base + d.n;
        data = d.data;
        offsets = d.offsets;
        part_base = d.part_base;
        partitions = d.partitions;
    }
};

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(kFullMask, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Exclusive prefix of cnt[0, count) into off[0, count), count <= kPartThreads * 8;
// every thread of the block calls it.  `warp_sums` has kPartThreads / 32 words.
__device__ __forceinline__ void block_exclusive_scan(const uint32_t *cnt, uint32_t *off, uint32_t count,
                                                     uint32_t *warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kPartThreads / 32;
    const uint32_t first = threadIdx.x * 8;
    uint32_t v[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        v[j] = first + j < count ? cnt[first + j] : 0u;
        sum += v[j];
    }
    const uint32_t incl = warp_incl_scan(sum, lane);
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? warp_sums[lane] : 0u;
        uint32_t wi = warp_incl_scan(w, lane);
        if (lane < kWarps) warp_sums[lane] = wi - w;
    }
    __syncthreads();
    uint32_t run = warp_sums[warp] + incl - sum;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        if (first + j < count) off[first + j] = run;
        run += v[j];
    }
    __syncthreads();
}

}  // namespace

static_assert(kMaxBins == (uint32_t)kPartThreads, "k_bin gives every thread at most one bin cursor");

size_t part_smem_bytes() { return sizeof(uint4) * kPartTile; }

// Pass 1.  Shared memory: fulcrums (static), bin counters and bases (static),
// the staged tile (dynamic).
template <int KIND>
__global__ void __launch_bounds__(kPartThreads, 2) k_bin(MapArgs a, PartArgs p) {
    __shared__ uint32_t sf[kFulcrums];
    __shared__ uint32_t hist[kMaxBins], loff[kMaxBins], gbase[kMaxBins];
    __shared__ uint32_t warp_sums[kPartThreads / 32];
    extern __shared__ __align__(16) uint4 stage[];
    constexpr bool kReadMapped = KIND == PHOBIC_KEYS_STRINGS;
    if (!kReadMapped)
        for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = a.fulcs[i];
    const uint64_t tiles = (a.total_keys + kPartTile - 1) / kPartTile;
    SetCache sc;
    // u64 keys of one set (the plain build): partition ids need no set lookup.
    const bool raw_u64 = KIND == PHOBIC_KEYS_U64 && a.nsets == 1;
    const unsigned long long *keys64 = static_cast<const unsigned long long *>(a.sets[0].data);
    const uint32_t parts0 = a.sets[0].partitions;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t t0 = t * kPartTile;
        const uint32_t count = (uint32_t)(a.total_keys - t0 < (uint64_t)kPartTile ? a.total_keys - t0 : kPartTile);
        for (uint32_t i = threadIdx.x; i < p.nbins; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        uint4 rec[kPartItems];
        uint32_t rank[kPartItems];
        if (raw_u64) {
            // All of the tile's key loads of this thread are issued before any key is hashed.
            unsigned long long raw[kPartItems];
#pragma unroll
            for (int j = 0; j < kPartItems; j++) {
                const uint32_t q = j * kPartThreads + threadIdx.x;
                raw[j] = q < count ? __ldg(keys64 + t0 + q) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < kPartItems; j++) {
                const uint32_t q = j * kPartThreads + threadIdx.x;
                rank[j] = 0xFFFFFFFFu;
                if (q >= count) continue;
                const Key4 k = key_from_hash(xxh3::hash_u64(raw[j]));
                rec[j] = make_uint4(k.lower1, k.lower2, partition_of(k.partitioner, parts0), bucket_of(k.bucketer, sf));
                if (PHB_CHECK((rec[j].z >> p.wshift) < p.nbins)) rank[j] = atomicAdd(&hist[rec[j].z >> p.wshift], 1u);
            }
        } else {
#pragma unroll
        for (int j = 0; j < kPartItems; j++) {
            const uint32_t q = j * kPartThreads + threadIdx.x;
            rank[j] = 0xFFFFFFFFu;
            if (q >= count) continue;
            const uint64_t g = t0 + q;
            if constexpr (kReadMapped) {
                uint4 r = a.mapped[g];  // {gp, bucket, lower1, lower2}
                rec[j] = make_uint4(r.z, r.w, r.x, r.y);
            } else {
                sc.locate(a, g);
                Key4 k = load_key<KIND>(sc.data, sc.offsets, g - sc.lo);
                rec[j] = make_uint4(k.lower1, k.lower2, sc.part_base + partition_of(k.partitioner, sc.partitions),
                                    bucket_of(k.bucketer, sf));
            }
            if (PHB_CHECK((rec[j].z >> p.wshift) < p.nbins)) rank[j] = atomicAdd(&hist[rec[j].z >> p.wshift], 1u);
        }
        }
        __syncthreads();
        block_exclusive_scan(hist, loff, p.nbins, warp_sums);
        // Thread b takes bin b's cursor (kMaxBins == kPartThreads); the atomic's result is
        // used only after this thread's stage writes, which run while it is in flight.
        const uint32_t my_bin = threadIdx.x;
        const bool has_bin = my_bin < p.nbins && hist[my_bin] != 0;
        const uint32_t my_cur = has_bin ? atomicAdd(&p.bincur[my_bin], hist[my_bin]) : 0u;
#pragma unroll
        for (int j = 0; j < kPartItems; j++)
            if (rank[j] != 0xFFFFFFFFu && PHB_CHECK(loff[rec[j].z >> p.wshift] + rank[j] < (uint32_t)kPartTile))
                stage[loff[rec[j].z >> p.wshift] + rank[j]] = rec[j];
        if (has_bin) gbase[my_bin] = my_cur - loff[my_bin];
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < count; q += blockDim.x) {
            const uint4 r = stage[q];
            const uint64_t dst = (uint64_t)gbase[r.z >> p.wshift] + q;
            // dst >= total only when counts and keys disagree (the keys changed; K4 reports
            // it): the clamp keeps that store inside the array.
            if (PHB_CHECK(dst < a.total_keys)) p.inter[min(dst, a.total_keys - 1)] = r;
        }
        __syncthreads();
    }
}

// Pass 2.
__global__ void __launch_bounds__(kPartThreads, 2) k_place(PartArgs p, uint64_t total, uint2 *lowers, uint16_t *bkt) {
    __shared__ uint32_t hist[kLocalRange], base[kLocalRange];
    __shared__ uint32_t warp_sums[kPartThreads / 32];
    __shared__ uint32_t s_min, s_max;
    extern __shared__ __align__(16) uint4 stage[];
    const uint64_t tiles = (total + kPartTile - 1) / kPartTile;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t t0 = t * kPartTile;
        const uint32_t count = (uint32_t)(total - t0 < (uint64_t)kPartTile ? total - t0 : kPartTile);
        if (threadIdx.x == 0) s_min = 0xFFFFFFFFu, s_max = 0;
        __syncthreads();
        uint4 rec[kPartItems];
        uint32_t lo = 0xFFFFFFFFu, hi = 0;
#pragma unroll
        for (int j = 0; j < kPartItems; j++) {
            const uint32_t q = j * kPartThreads + threadIdx.x;
            if (q >= count) continue;
            rec[j] = p.inter[t0 + q];
            lo = min(lo, rec[j].z);
            hi = max(hi, rec[j].z);
        }
        lo = __reduce_min_sync(kFullMask, lo);
        hi = __reduce_max_sync(kFullMask, hi);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_min, lo);
            atomicMax(&s_max, hi);
        }
        __syncthreads();
        const uint32_t gmin = s_min, range = s_max - s_min + 1;
        if (s_max >= p.M) {  // a record of no partition: pass 1 left it unwritten (the keys changed)
            (void)PHB_CHECK(false);
            __syncthreads();
            continue;
        }
        if (range > kLocalRange) {  // partitions too small for runs: one atomic per record
#pragma unroll
            for (int j = 0; j < kPartItems; j++) {
                const uint32_t q = j * kPartThreads + threadIdx.x;
                if (q >= count) continue;
                const uint32_t dst = (uint32_t)min((uint64_t)atomicAdd(&p.pcur[rec[j].z], 1u), total - 1);
                if (!PHB_CHECK(dst < total)) continue;
                lowers[dst] = make_uint2(rec[j].x, rec[j].y);
                bkt[dst] = (uint16_t)rec[j].w;
            }
            __syncthreads();
            continue;
        }
        for (uint32_t i = threadIdx.x; i < range; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        uint32_t rank[kPartItems];
#pragma unroll
        for (int j = 0; j < kPartItems; j++) {
            const uint32_t q = j * kPartThreads + threadIdx.x;
            rank[j] = q < count ? atomicAdd(&hist[rec[j].z - gmin], 1u) : 0xFFFFFFFFu;
        }
        __syncthreads();
        block_exclusive_scan(hist, base, range, warp_sums);  // base = local offsets
        // Partition cursors: thread i's first partition's atomic is issued before its stage
        // writes and used after them; hist[i] becomes the global base of partition
        // gmin + i less its local offset (hist is free once the scan has read it).
        const uint32_t i0 = threadIdx.x;
        const bool has0 = i0 < range && hist[i0] != 0;
        const uint32_t cur0 = has0 ? atomicAdd(&p.pcur[gmin + i0], hist[i0]) : 0u;
#pragma unroll
        for (int j = 0; j < kPartItems; j++)
            if (rank[j] != 0xFFFFFFFFu && PHB_CHECK(base[rec[j].z - gmin] + rank[j] < (uint32_t)kPartTile))
                stage[base[rec[j].z - gmin] + rank[j]] = rec[j];
        if (has0) hist[i0] = cur0 - base[i0];
        for (uint32_t i = i0 + blockDim.x; i < range; i += blockDim.x)
            if (hist[i]) hist[i] = atomicAdd(&p.pcur[gmin + i], hist[i]) - base[i];
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < count; q += blockDim.x) {
            const uint4 r = stage[q];
            // Clamped: only a build whose keys changed (reported by K4) gets past total.
            const uint32_t dst = (uint32_t)min((uint64_t)(hist[r.z - gmin] + q), total - 1);
            if (!PHB_CHECK(dst < total)) continue;
            lowers[dst] = make_uint2(r.x, r.y);
            bkt[dst] = (uint16_t)r.w;
        }
        __syncthreads();
    }
}

unsigned int check_line_part(bool reset) { return read_check_line(reset); }

uint32_t part_wshift(uint64_t partitions) {
    uint32_t w = 0;
    while (((partitions + (1ull << w) - 1) >> w) > kTargetBins) w++;
    // A pass-2 tile spans at most two bins; keep that within kLocalRange partition ids
    // (else pass 2 places its records one atomic at a time) as long as the bins fit
    // kMaxBins.
    while ((2ull << w) > kLocalRange && w > 0 && ((partitions + (1ull << (w - 1)) - 1) >> (w - 1)) <= kMaxBins) w--;
    return w;
}

template <int KIND>
static cudaError_t launch_bin_kind(const MapArgs &a, const PartArgs &p, int grid, cudaStream_t st) {
    const size_t smem = part_smem_bytes();
    cudaError_t e = allow_dynamic_smem(k_bin<KIND>, smem);
    if (e != cudaSuccess) return e;
    k_bin<KIND><<<grid, kPartThreads, smem, st>>>(a, p);
    return cudaGetLastError();
}

cudaError_t launch_partition(int kind, const MapArgs &a, const PartArgs &p, int sm_count, cudaStream_t st) {
    if (a.total_keys == 0) return cudaSuccess;
    const uint64_t tiles = (a.total_keys + kPartTile - 1) / kPartTile;
    const uint64_t cap = (uint64_t)(sm_count > 0 ? sm_count : 148) * 2;
    const int grid = (int)(tiles < cap ? tiles : cap);
    cudaError_t e;
    switch (kind) {
    case PHOBIC_KEYS_U64: e = launch_bin_kind<PHOBIC_KEYS_U64>(a, p, grid, st); break;
    case PHOBIC_KEYS_BYTES16: e = launch_bin_kind<PHOBIC_KEYS_BYTES16>(a, p, grid, st); break;
    case PHOBIC_KEYS_PREHASHED: e = launch_bin_kind<PHOBIC_KEYS_PREHASHED>(a, p, grid, st); break;
    default: e = launch_bin_kind<PHOBIC_KEYS_STRINGS>(a, p, grid, st); break;
    }
    if (e != cudaSuccess) return e;
    const size_t smem = part_smem_bytes();
    e = allow_dynamic_smem(k_place, smem);
    if (e != cudaSuccess) return e;
    k_place<<<grid, kPartThreads, smem, st>>>(p, a.total_keys, a.lowers, a.bkt);
    return cudaGetLastError();
}

}  // namespace phobicb200
