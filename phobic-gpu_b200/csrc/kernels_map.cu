// K1 (map_count) and K3 (scatter): the streaming stages of the build.
//
// K1 replaces the host initial hash (include/phobicGpu/mphf_builder.h:201-216)
// and the bucket_sizes stage (shaders/bucket_sizes.comp:21-35): every key is
// hashed with XXH3-128 on the device, mapped to its partition
// (key_mapping.glsl:43-45) and bucket (:34-41), and counted per partition.
//
// K3 replaces apply_partition_offset.comp:9-18 and redistribute_keys.comp:21-53:
// each key's (lower1, lower2) pair and bucket id are appended to its partition
// through one of the partition's kSub cursors (chosen by the key index) that K2
// set to the start of that cursor's slot range.  Appending in arrival order keeps
// every write front inside one or two L2 sectors, so the scattered 8-byte and
// 2-byte stores merge in L2 before they reach HBM; spreading a partition over
// kSub cursors keeps same-address atomics from queueing behind each other.  The bucket order inside a partition is produced later, in
// shared memory, by K4.
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
constexpr int kUnroll = 4;

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
            if constexpr (kReadMapped) {
                uint4 r = a.mapped[g];
                gp[u] = r.x, b[u] = r.y, l1[u] = r.z, l2[u] = r.w;
            } else {
                c.locate(a, g);
                Key4 k = load_key<KIND>(c.data, c.offsets, g - c.lo);
                gp[u] = c.part_base + partition_of(k.partitioner, c.partitions);
                b[u] = bucket_of(k.bucketer, sf);
                l1[u] = k.lower1, l2[u] = k.lower2;
                if (!SCATTER) {
                    if (b[u] >= a.buckets && bad_set == 0xFFFFFFFFu) bad_set = c.s;
                    if (a.debug_keys) a.debug_keys[g] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
                }
            }
        }
        if constexpr (SCATTER) {
            uint32_t slot[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++)
                if (gp[u] != 0xFFFFFFFFu)
                    slot[u] = atomicAdd(&a.counts[(size_t)gp[u] * kSub + ((g0 + u * stride) & (kSub - 1))], 1u);
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu) continue;
                a.lowers[slot[u]] = make_uint2(l1[u], l2[u]);
                a.bkt[slot[u]] = (uint16_t)b[u];
            }
        } else {
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                if (gp[u] == 0xFFFFFFFFu) continue;
                atomicAdd(&a.counts[(size_t)gp[u] * kSub + ((g0 + u * stride) & (kSub - 1))], 1u);
                if (KIND == PHOBIC_KEYS_STRINGS) a.mapped[g0 + u * stride] = make_uint4(gp[u], b[u], l1[u], l2[u]);
            }
        }
    }
    if (bad_set != 0xFFFFFFFFu) report_error(&a.err[bad_set], 0, PHOBIC_ERR_INVALID);
}

template <bool SCATTER>
static cudaError_t launch_map(int kind, const MapArgs &a, int grid, cudaStream_t st) {
    if (a.total_keys == 0) return cudaSuccess;
    switch (kind) {
    case PHOBIC_KEYS_U64: k_map<PHOBIC_KEYS_U64, SCATTER><<<grid, kMapThreads, 0, st>>>(a); break;
    case PHOBIC_KEYS_BYTES16: k_map<PHOBIC_KEYS_BYTES16, SCATTER><<<grid, kMapThreads, 0, st>>>(a); break;
    case PHOBIC_KEYS_PREHASHED: k_map<PHOBIC_KEYS_PREHASHED, SCATTER><<<grid, kMapThreads, 0, st>>>(a); break;
    default: k_map<PHOBIC_KEYS_STRINGS, SCATTER><<<grid, kMapThreads, 0, st>>>(a); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_map_count(int kind, const MapArgs &a, int grid, cudaStream_t st) {
    return launch_map<false>(kind, a, grid, st);
}

cudaError_t launch_scatter(int kind, const MapArgs &a, int grid, cudaStream_t st) {
    return launch_map<true>(kind, a, grid, st);
}

}  // namespace phobicb200
