// K1 (map_count) and K3 (scatter): the streaming stages of the build.
//
// K1 replaces the host initial hash (include/phobicGpu/mphf_builder.h:201-216)
// and the bucket_sizes stage (shaders/bucket_sizes.comp:21-35): every key is
// hashed with XXH3-128 on the device, mapped to its partition
// (key_mapping.glsl:43-45) and bucket (:34-41), and counted per partition.
//
// K3 replaces apply_partition_offset.comp:9-18 and redistribute_keys.comp:21-53:
// each key's (lower1, lower2) pair and bucket id are appended to its partition.
// The bucket order inside a partition is produced later, in shared memory, by K4.
//
// Two plans (plan_map):
//   chunked  CTA c counts (K1) and places (K3) the keys of one contiguous chunk
//            with a shared-memory counter per partition; the only global traffic
//            is the streamed keys, one column of the count matrix and the record
//            stores.  Used while all partitions' counters fit in shared memory,
//            32-bit up to 52K partitions, packed 16-bit (counting) up to 104K.
//   global   one counter per partition in global memory, a reduction per key in
//            K1 and an atomic add per key in K3 (builds with more partitions).
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

}  // namespace

// Each thread takes kUnroll keys per iteration, kStride apart, so that their
// loads and atomics are in flight together; the warp's loads stay coalesced.
constexpr int kUnroll = 8;

// Partition, bucket and lower pair of global key g.
template <int KIND, bool READ_MAPPED>
__device__ __forceinline__ void map_key(const MapArgs &a, SetCache &c, const uint32_t *sf, uint64_t g, uint32_t &gp,
                                        uint32_t &b, uint32_t &l1, uint32_t &l2) {
    if constexpr (READ_MAPPED) {
        uint4 r = a.mapped[g];
        gp = r.x, b = r.y, l1 = r.z, l2 = r.w;
    } else {
        c.locate(a, g);
        Key4 k = load_key<KIND>(c.data, c.offsets, g - c.lo);
        gp = c.part_base + partition_of(k.partitioner, c.partitions);
        b = bucket_of(k.bucketer, sf);
        l1 = k.lower1, l2 = k.lower2;
    }
}

// Global plan: grid-stride over all keys, one global counter per partition.
template <int KIND, bool SCATTER>
__global__ void __launch_bounds__(kMapThreads) k_map(MapArgs a) {
    __shared__ uint32_t sf[kFulcrums];
    constexpr bool kReadMapped = SCATTER && KIND == PHOBIC_KEYS_STRINGS;
    if (!kReadMapped) {
        for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = a.fulcs[i];
        __syncthreads();
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    SetCache c;
    uint32_t bad_set = 0xFFFFFFFFu;
    for (uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g0 < a.total_keys; g0 += kUnroll * stride) {
        uint32_t gp[kUnroll], b[kUnroll], l1[kUnroll], l2[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const uint64_t g = g0 + u * stride;
            gp[u] = 0xFFFFFFFFu;
            if (g >= a.total_keys) continue;
            map_key<KIND, kReadMapped>(a, c, sf, g, gp[u], b[u], l1[u], l2[u]);
            if (!SCATTER) {
                if (b[u] >= a.buckets && bad_set == 0xFFFFFFFFu) bad_set = c.s;
                if (a.debug_keys) {
                    Key4 k = load_key<KIND>(c.data, c.offsets, g - c.lo);
                    a.debug_keys[g] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
                }
            }
        }
        if constexpr (SCATTER) {
            uint32_t slot[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++)
                if (gp[u] != 0xFFFFFFFFu) slot[u] = PHB_CHECK(gp[u] < a.M) ? atomicAdd(&a.counts[gp[u]], 1u) : 0u;
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu) continue;
                // A slot at or past the end only comes from keys that changed since K1 counted
                // them (the search reports PHOBIC_ERR_KEYS_CHANGED): the clamp keeps the store in
                // the record arrays.
                const uint64_t at = slot[u] < a.total_keys ? slot[u] : a.total_keys - 1;
                if (!PHB_CHECK(slot[u] < a.total_keys)) continue;
                a.lowers[at] = make_uint2(l1[u], l2[u]);
                a.bkt[at] = (uint16_t)b[u];
            }
        } else {
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu) continue;
                atomicAdd(&a.counts[gp[u]], 1u);
                if (KIND == PHOBIC_KEYS_STRINGS) a.mapped[g0 + u * stride] = make_uint4(gp[u], b[u], l1[u], l2[u]);
            }
        }
    }
    if (bad_set != 0xFFFFFFFFu) report_error(&a.err[bad_set], 0, PHOBIC_ERR_INVALID);
}

// A 16-bit counter of the packed plan went from 0xFFFF to 0 in the add that
// returned `old`: credit the 65536 keys to column c of the count matrix.  The
// half-word arithmetic is exact because each half only ever steps by one: a low
// half (even partition g) that wraps carries one into the high half (g + 1),
// which is taken back here, and if that carry wrapped the high half too, the
// high half's 65536 is credited as well.  An odd partition's wrap carries out of
// the word.  Rare by construction: it takes 65536 keys of one partition in one
// chunk, and the build then fails its size check (partitions hold <= 65535 keys).
static __device__ __forceinline__ void credit_wrap(const MapArgs &a, uint32_t c, uint32_t g, uint32_t old, uint32_t *wrapped) {
    *wrapped = 1u;
    atomicAdd(&a.counts[(size_t)g * a.stride + c], 65536u);
    if ((g & 1u) == 0 && g + 1 < a.M)
        atomicAdd(&a.counts[(size_t)(g + 1) * a.stride + c], (old >> 16) == 0xFFFFu ? 65535u : 0xFFFFFFFFu);
}

// Chunked plan: CTA c owns keys [c * chunk, (c + 1) * chunk).  K1 counts them per
// partition in shared memory and writes column c of the count matrix; K3 loads
// column c of its exclusive scan as cursors and hands out slots with
// shared-memory atomics.  NARROW (K1 only) packs two 16-bit counters per word.
template <int KIND, bool SCATTER, bool NARROW>
__global__ void __launch_bounds__(kChunkThreads, 1) k_chunk(MapArgs a) {
    static_assert(!(SCATTER && NARROW), "slots need 32-bit cursors");
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t wrapped;       // a 16-bit counter wrapped in this CTA
    uint32_t *sf = smem;               // [kFulcrums]
    uint32_t *cnt = smem + kFulcrums;  // [M], or [(M + 1) / 2] packed
    constexpr bool kReadMapped = SCATTER && KIND == PHOBIC_KEYS_STRINGS;
    const uint32_t c = blockIdx.x;
    if (!kReadMapped)
        for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = a.fulcs[i];
    const uint32_t words = NARROW ? (a.M + 1) / 2 : a.M;
    for (uint32_t g = threadIdx.x; g < words; g += blockDim.x) cnt[g] = SCATTER ? a.counts[(size_t)g * a.stride + c] : 0u;
    if (threadIdx.x == 0) wrapped = 0u;
    __syncthreads();

    const uint64_t lo = (uint64_t)c * a.chunk;
    const uint64_t hi = lo + a.chunk < a.total_keys ? lo + a.chunk : a.total_keys;
    SetCache sc;
    uint32_t bad_set = 0xFFFFFFFFu;
    // u64 keys of one set (the plain build): all of an iteration's key loads are
    // issued before any of them is hashed, so kUnroll loads per thread are in flight.
    constexpr bool kRawU64 = KIND == PHOBIC_KEYS_U64 && !kReadMapped;
    const bool raw_u64 = kRawU64 && a.nsets == 1;
    const unsigned long long *keys64 = kRawU64 ? static_cast<const unsigned long long *>(a.sets[0].data) : nullptr;
    const uint32_t parts0 = a.sets[0].partitions;
    for (uint64_t g0 = lo + threadIdx.x; g0 < hi; g0 += (uint64_t)kUnroll * kChunkThreads) {
        uint32_t gp[kUnroll], b[kUnroll], l1[kUnroll], l2[kUnroll];
        if (raw_u64) {
            uint64_t raw[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const uint64_t g = g0 + (uint64_t)u * kChunkThreads;
                raw[u] = g < hi ? __ldg(keys64 + g) : 0ull;
            }
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const uint64_t g = g0 + (uint64_t)u * kChunkThreads;
                gp[u] = 0xFFFFFFFFu;
                if (g >= hi) continue;
                const Key4 k = key_from_hash(xxh3::hash_u64(raw[u]));
                gp[u] = partition_of(k.partitioner, parts0);
                b[u] = bucket_of(k.bucketer, sf);
                l1[u] = k.lower1, l2[u] = k.lower2;
                if (!SCATTER) {
                    if (b[u] >= a.buckets && bad_set == 0xFFFFFFFFu) bad_set = 0;
                    if (a.debug_keys) a.debug_keys[g] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
                }
            }
        } else {
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const uint64_t g = g0 + (uint64_t)u * kChunkThreads;
            gp[u] = 0xFFFFFFFFu;
            if (g >= hi) continue;
            map_key<KIND, kReadMapped>(a, sc, sf, g, gp[u], b[u], l1[u], l2[u]);
            if (!SCATTER) {
                if (b[u] >= a.buckets && bad_set == 0xFFFFFFFFu) bad_set = sc.s;
                if (a.debug_keys) {
                    Key4 k = load_key<KIND>(sc.data, sc.offsets, g - sc.lo);
                    a.debug_keys[g] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
                }
            }
        }
        }
        if constexpr (SCATTER) {
            uint32_t slot[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++)
                if (gp[u] != 0xFFFFFFFFu) slot[u] = PHB_CHECK(gp[u] < a.M) ? atomicAdd(&cnt[gp[u]], 1u) : 0u;
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu) continue;
                a.lowers[slot[u]] = make_uint2(l1[u], l2[u]);
                a.bkt[slot[u]] = (uint16_t)b[u];
            }
        } else if constexpr (NARROW) {
            uint32_t old[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                old[u] = 0u;
                if (gp[u] == 0xFFFFFFFFu || !PHB_CHECK(gp[u] < a.M)) continue;
                old[u] = atomicAdd(&cnt[gp[u] >> 1], 1u << ((gp[u] & 1u) << 4));
                if (KIND == PHOBIC_KEYS_STRINGS)
                    a.mapped[g0 + (uint64_t)u * kChunkThreads] = make_uint4(gp[u], b[u], l1[u], l2[u]);
            }
#pragma unroll
            for (int u = 0; u < kUnroll; u++)
                if (gp[u] < a.M && ((old[u] >> ((gp[u] & 1u) << 4)) & 0xFFFFu) == 0xFFFFu)
                    credit_wrap(a, c, gp[u], old[u], &wrapped);
        } else {
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu || !PHB_CHECK(gp[u] < a.M)) continue;
                atomicAdd(&cnt[gp[u]], 1u);
                if (KIND == PHOBIC_KEYS_STRINGS)
                    a.mapped[g0 + (uint64_t)u * kChunkThreads] = make_uint4(gp[u], b[u], l1[u], l2[u]);
            }
        }
    }
    if (bad_set != 0xFFFFFFFFu) report_error(&a.err[bad_set], 0, PHOBIC_ERR_INVALID);
    if (!SCATTER) {
        __syncthreads();
        if (NARROW) {
            // After a wrap the column already holds the credited 65536s: add to it.
            const bool add = wrapped != 0u;
            for (uint32_t g = threadIdx.x; g < a.M; g += blockDim.x) {
                const uint32_t v = (cnt[g >> 1] >> ((g & 1u) << 4)) & 0xFFFFu;
                if (add)
                    atomicAdd(&a.counts[(size_t)g * a.stride + c], v);
                else
                    a.counts[(size_t)g * a.stride + c] = v;
            }
        } else {
            for (uint32_t g = threadIdx.x; g < a.M; g += blockDim.x) a.counts[(size_t)g * a.stride + c] = cnt[g];
        }
    }
}

// K1 for string keys, with coalesced loads of the ragged bytes.  A warp takes 32
// consecutive strings of one set at a time: their bytes are one contiguous span of
// the set's data, which the warp copies into its shared-memory stage with 16-byte
// loads (byte loads only for the unaligned head and tail, so no load leaves the
// span), and each lane then hashes its own string from the stage.  A group whose
// span does not fit the stage, or whose strings belong to two sets, is hashed from
// global memory as before.  Counting, the bucket-id check and the {partition,
// bucket, lower1, lower2} records for K3 are those of k_chunk.
constexpr uint32_t kStrStageBytes = 2304;  // per warp: 32 strings of up to 64 bytes, with slack
constexpr uint32_t kStrStageSlack = 32;    // alignment (<= 15 bytes) and the stage reads' overhang (<= 12)

// The stage as a byte source for the hash: bytes [start, start + len) of the warp's
// stage, read with 32-bit shared-memory loads and funnel shifts.
struct StageSrc {
    uint32_t sa;     // shared-space byte address of the stage
    uint32_t start;  // the string's first byte inside the stage

    __device__ __forceinline__ uint32_t word(uint32_t k) const {
        uint32_t v;
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(sa + 4 * k));
        return v;
    }
    __device__ __forceinline__ uint8_t b(size_t i) const {
        const uint32_t x = start + (uint32_t)i;
        return (uint8_t)(word(x >> 2) >> ((x & 3) * 8));
    }
    __device__ __forceinline__ uint32_t r32(size_t i) const {
        const uint32_t x = start + (uint32_t)i, k = x >> 2, sh = (x & 3) * 8;
        return __funnelshift_r(word(k), word(k + 1), sh);
    }
    __device__ __forceinline__ uint64_t r64(size_t i) const {
        const uint32_t x = start + (uint32_t)i, k = x >> 2, sh = (x & 3) * 8;
        const uint32_t w0 = word(k), w1 = word(k + 1), w2 = word(k + 2);
        return (uint64_t)__funnelshift_r(w0, w1, sh) | ((uint64_t)__funnelshift_r(w1, w2, sh) << 32);
    }
};

template <bool NARROW>
__global__ void __launch_bounds__(kChunkThreads, 1) k_chunk_str(MapArgs a) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t wrapped;
    uint32_t *sf = smem;               // [kFulcrums]
    uint32_t *cnt = smem + kFulcrums;  // [M], or [(M + 1) / 2] packed
    const uint32_t words = NARROW ? (a.M + 1) / 2 : a.M;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *stage = smem + ((kFulcrums + words + 3) & ~3u) + (size_t)warp * (kStrStageBytes / 4);
    const uint32_t stage_sa = (uint32_t)__cvta_generic_to_shared(stage);
    char *stage_b = reinterpret_cast<char *>(stage);
    const uint32_t c = blockIdx.x;
    for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = a.fulcs[i];
    for (uint32_t g = threadIdx.x; g < words; g += blockDim.x) cnt[g] = 0u;
    if (threadIdx.x == 0) wrapped = 0u;
    __syncthreads();

    const uint64_t lo = (uint64_t)c * a.chunk;
    const uint64_t hi = lo + a.chunk < a.total_keys ? lo + a.chunk : a.total_keys;
    SetCache sc;
    uint32_t bad_set = 0xFFFFFFFFu;
    constexpr uint64_t kGroupStride = 32 * (uint64_t)(kChunkThreads / 32);
    // The next group's offsets are loaded while the current group is staged and hashed
    // (when they lie in the set of the current lane's key), so a group waits for one
    // round trip to memory (its bytes), not two (offsets, then bytes).
    bool have_next = false;
    uint64_t a_next = 0, b_next = 0;
    for (uint64_t gbase = lo + 32 * (uint64_t)warp; gbase < hi; gbase += kGroupStride) {
        const uint64_t g = gbase + lane;
        const bool valid = g < hi;
        uint64_t a_off = 0, b_off = 0;
        if (valid) {
            if (have_next) {
                a_off = a_next;
                b_off = b_next;
            } else {
                sc.locate(a, g);
                a_off = __ldg(reinterpret_cast<const unsigned long long *>(sc.offsets) + (g - sc.lo));
                b_off = __ldg(reinterpret_cast<const unsigned long long *>(sc.offsets) + (g - sc.lo) + 1);
            }
        }
        const uint64_t gn = g + kGroupStride;
        have_next = valid && gn < hi && gn < sc.hi;  // same set as this lane's key: sc stays valid
        if (have_next) {
            a_next = __ldg(reinterpret_cast<const unsigned long long *>(sc.offsets) + (gn - sc.lo));
            b_next = __ldg(reinterpret_cast<const unsigned long long *>(sc.offsets) + (gn - sc.lo) + 1);
        }
        const uint32_t vmask = __ballot_sync(kFullMask, valid);
        const int last = 31 - __clz(vmask);
        const unsigned long long data0 = __shfl_sync(kFullMask, (unsigned long long)sc.data, 0);
        const bool one_set = __all_sync(kFullMask, !valid || (unsigned long long)sc.data == data0);
        const uint64_t span_lo = __shfl_sync(kFullMask, a_off, 0), span_hi = __shfl_sync(kFullMask, b_off, last);
        Key4 k{};
        if (one_set && span_hi >= span_lo && span_hi - span_lo <= kStrStageBytes - kStrStageSlack) {
            const uint64_t A = data0 + span_lo, E = data0 + span_hi;
            const uint64_t A0 = A & ~15ull, A16 = (A + 15) & ~15ull, E16 = E & ~15ull;
            // Interior 16-byte blocks, then the head [A, min(A16, E)) and the tail
            // [max(E16, A16), E): every load lies inside [A, E).
            for (uint64_t q = A16 + 16 * (uint64_t)lane; q + 16 <= E16; q += 512)
                *reinterpret_cast<uint4 *>(stage_b + (q - A0)) = __ldg(reinterpret_cast<const uint4 *>(q));
            const uint64_t head_end = A16 < E ? A16 : E, tail_begin = E16 > A16 ? E16 : A16;
            if (A + lane < head_end) stage_b[A + lane - A0] = (char)__ldg(reinterpret_cast<const unsigned char *>(A + lane));
            if (tail_begin + lane < E)
                stage_b[tail_begin + lane - A0] = (char)__ldg(reinterpret_cast<const unsigned char *>(tail_begin + lane));
            __syncwarp();
            if (valid)
                k = key_from_hash(xxh3::hash_src(StageSrc{stage_sa, (uint32_t)(A - A0 + (a_off - span_lo))},
                                                 (size_t)(b_off - a_off)));
            __syncwarp();
        } else if (valid) {
            k = key_from_hash(xxh3::hash_bytes(static_cast<const uint8_t *>(sc.data) + a_off, (size_t)(b_off - a_off)));
        }
        if (!valid) continue;
        const uint32_t gp = sc.part_base + partition_of(k.partitioner, sc.partitions);
        const uint32_t b = bucket_of(k.bucketer, sf);
        if (b >= a.buckets && bad_set == 0xFFFFFFFFu) bad_set = sc.s;
        if (a.debug_keys) a.debug_keys[g] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
        a.mapped[g] = make_uint4(gp, b, k.lower1, k.lower2);
        if (!PHB_CHECK(gp < a.M)) continue;
        if (NARROW) {
            const uint32_t old = atomicAdd(&cnt[gp >> 1], 1u << ((gp & 1u) << 4));
            if (((old >> ((gp & 1u) << 4)) & 0xFFFFu) == 0xFFFFu) credit_wrap(a, c, gp, old, &wrapped);
        } else {
            atomicAdd(&cnt[gp], 1u);
        }
    }
    if (bad_set != 0xFFFFFFFFu) report_error(&a.err[bad_set], 0, PHOBIC_ERR_INVALID);
    __syncthreads();
    if (NARROW) {
        const bool add = wrapped != 0u;
        for (uint32_t g = threadIdx.x; g < a.M; g += blockDim.x) {
            const uint32_t v = (cnt[g >> 1] >> ((g & 1u) << 4)) & 0xFFFFu;
            if (add)
                atomicAdd(&a.counts[(size_t)g * a.stride + c], v);
            else
                a.counts[(size_t)g * a.stride + c] = v;
        }
    } else {
        for (uint32_t g = threadIdx.x; g < a.M; g += blockDim.x) a.counts[(size_t)g * a.stride + c] = cnt[g];
    }
}

unsigned int check_line_map(bool reset) { return read_check_line(reset); }

static __global__ void k_change_key(unsigned long long *keys, uint64_t index, unsigned long long mask) {
    keys[index] ^= mask;
}

cudaError_t launch_change_key(void *keys, uint64_t index, uint64_t mask, cudaStream_t st) {
    k_change_key<<<1, 1, 0, st>>>(static_cast<unsigned long long *>(keys), index, mask);
    return cudaGetLastError();
}

static size_t chunk_smem(uint64_t partitions, bool narrow) {
    return 4 * ((size_t)kFulcrums + (size_t)(narrow ? (partitions + 1) / 2 : partitions));
}

MapPlan plan_map(uint64_t total_keys, uint64_t partitions, int sm_count) {
    MapPlan p{};
    if (partitions <= kChunkNarrowMaxPartitions && total_keys > 0) {
        uint64_t ctas = (total_keys + kChunkMinKeys - 1) / kChunkMinKeys;
        if (ctas > kChunkCtas) ctas = kChunkCtas;
        p.chunked = true;
        p.stride = (uint32_t)ctas;
        p.grid = (uint32_t)ctas;
        p.chunk = (total_keys + ctas - 1) / ctas;
        p.narrow = partitions > kChunkMaxPartitions;
    } else {
        p.chunked = false;
        p.stride = 1;
        uint64_t want = (total_keys + kMapThreads - 1) / kMapThreads;
        uint64_t cap = (uint64_t)(sm_count > 0 ? sm_count : 148) * 8;
        p.grid = (uint32_t)(want < cap ? (want ? want : 1) : cap);
        p.chunk = 0;
    }
    return p;
}

// Shared memory of k_chunk_str: the counters, then one stage per warp.
static size_t chunk_str_smem(uint64_t partitions, bool narrow) {
    const size_t words = (size_t)kFulcrums + (size_t)(narrow ? (partitions + 1) / 2 : partitions);
    return 4 * ((words + 3) & ~size_t(3)) + (size_t)(kChunkThreads / 32) * kStrStageBytes;
}

template <int KIND, bool SCATTER, bool NARROW>
static cudaError_t launch_chunk(const MapArgs &a, const MapPlan &plan, cudaStream_t st) {
    if constexpr (KIND == PHOBIC_KEYS_STRINGS && !SCATTER) {
        // Staged string loads whenever the stages fit beside the counters.
        const size_t smem = chunk_str_smem(a.M, NARROW);
        if (allow_dynamic_smem(k_chunk_str<NARROW>, smem) == cudaSuccess) {
            k_chunk_str<NARROW><<<plan.grid, kChunkThreads, smem, st>>>(a);
            return cudaSuccess;
        }
        cudaGetLastError();
    }
    const size_t smem = chunk_smem(a.M, NARROW);
    cudaError_t e = allow_dynamic_smem(k_chunk<KIND, SCATTER, NARROW>, smem);
    if (e != cudaSuccess) return e;
    k_chunk<KIND, SCATTER, NARROW><<<plan.grid, kChunkThreads, smem, st>>>(a);
    return cudaSuccess;
}

template <bool SCATTER, int KIND>
static cudaError_t launch_kind(const MapArgs &a, const MapPlan &plan, cudaStream_t st) {
    if (plan.chunked) {
        cudaError_t e;
        if constexpr (SCATTER)
            e = plan.narrow ? cudaErrorInvalidValue : launch_chunk<KIND, true, false>(a, plan, st);
        else
            e = plan.narrow ? launch_chunk<KIND, false, true>(a, plan, st) : launch_chunk<KIND, false, false>(a, plan, st);
        if (e != cudaSuccess) return e;
    } else {
        k_map<KIND, SCATTER><<<plan.grid, kMapThreads, 0, st>>>(a);
    }
    return cudaGetLastError();
}

template <bool SCATTER>
static cudaError_t launch_map(int kind, const MapArgs &a, const MapPlan &plan, cudaStream_t st) {
    if (a.total_keys == 0) return cudaSuccess;
    switch (kind) {
    case PHOBIC_KEYS_U64: return launch_kind<SCATTER, PHOBIC_KEYS_U64>(a, plan, st);
    case PHOBIC_KEYS_BYTES16: return launch_kind<SCATTER, PHOBIC_KEYS_BYTES16>(a, plan, st);
    case PHOBIC_KEYS_PREHASHED: return launch_kind<SCATTER, PHOBIC_KEYS_PREHASHED>(a, plan, st);
    default: return launch_kind<SCATTER, PHOBIC_KEYS_STRINGS>(a, plan, st);
    }
}

cudaError_t launch_map_count(int kind, const MapArgs &a, const MapPlan &plan, cudaStream_t st) {
    return launch_map<false>(kind, a, plan, st);
}

cudaError_t launch_scatter(int kind, const MapArgs &a, const MapPlan &plan, cudaStream_t st) {
    return launch_map<true>(kind, a, plan, st);
}

}  // namespace phobicb200
