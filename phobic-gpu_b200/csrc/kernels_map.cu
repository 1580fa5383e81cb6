// K1 (map_count) and K3 (scatter): the streaming stages of the build.
//
// K1 replaces the host initial hash (include/phobicGpu/mphf_builder.h:201-216)
// and the bucket_sizes stage (shaders/bucket_sizes.comp:21-35): every key is
// hashed with XXH3-128 on the device, mapped to its partition
// (key_mapping.glsl:43-45) and bucket (:34-41), and counted per partition; the
// count returned by the atomic is the key's rank inside its partition.
//
// K3 replaces apply_partition_offset.comp:9-18 and redistribute_keys.comp:21-53:
// each key's (lower1, lower2) pair and bucket id land at
// partition_offset[p] + rank, which makes every partition contiguous.  The
// bucket order inside a partition is produced later in shared memory by K4.
#include "kernels.cuh"

namespace phobicb200 {

__device__ __forceinline__ void load_fulcrums(uint32_t *sf, const uint32_t *fulcs) {
    for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = fulcs[i];
    __syncthreads();
}

template <int KIND>
__global__ void __launch_bounds__(kMapThreads) k_map_count(KeyInput in, uint64_t n, MapArgs a) {
    __shared__ uint32_t sf[kFulcrums];
    load_fulcrums(sf, a.fulcs);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool bad = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Key4 k = load_key<KIND>(in, i);
        uint32_t p = partition_of(k.partitioner, a.partitions);
        uint32_t b = bucket_of(k.bucketer, sf);
        bad |= b >= a.buckets;
        a.rank[i] = atomicAdd(&a.part_count[p], 1u);
        if (a.mapped) a.mapped[i] = make_uint4(p, b, k.lower1, k.lower2);
        if (a.debug_keys) a.debug_keys[i] = make_uint4(k.partitioner, k.bucketer, k.lower1, k.lower2);
    }
    if (bad) report_error(a.err, 0, PHOBIC_ERR_INVALID);
}

template <int KIND>
__global__ void __launch_bounds__(kMapThreads) k_scatter(KeyInput in, uint64_t n, ScatterArgs a) {
    __shared__ uint32_t sf[kFulcrums];
    if (!a.mapped) load_fulcrums(sf, a.fulcs);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t p, b, l1, l2;
        if (a.mapped) {
            uint4 r = a.mapped[i];
            p = r.x, b = r.y, l1 = r.z, l2 = r.w;
        } else {
            Key4 k = load_key<KIND>(in, i);
            p = partition_of(k.partitioner, a.partitions);
            b = bucket_of(k.bucketer, sf);
            l1 = k.lower1, l2 = k.lower2;
        }
        uint32_t dst = a.part_off[p] + a.rank[i];
        a.lowers[dst] = make_uint2(l1, l2);
        a.bkt[dst] = (uint16_t)b;
    }
}

template <int KIND>
static cudaError_t launch_map_kind(const KeyInput &in, uint64_t n, const MapArgs &m, const ScatterArgs &s, int grid,
                                   cudaStream_t st, bool scatter) {
    if (scatter) k_scatter<KIND><<<grid, kMapThreads, 0, st>>>(in, n, s);
    else k_map_count<KIND><<<grid, kMapThreads, 0, st>>>(in, n, m);
    return cudaGetLastError();
}

cudaError_t launch_map_count(int kind, const KeyInput &in, uint64_t n, const MapArgs &a, int grid, cudaStream_t st) {
    ScatterArgs none{};
    switch (kind) {
    case PHOBIC_KEYS_U64: return launch_map_kind<PHOBIC_KEYS_U64>(in, n, a, none, grid, st, false);
    case PHOBIC_KEYS_BYTES16: return launch_map_kind<PHOBIC_KEYS_BYTES16>(in, n, a, none, grid, st, false);
    case PHOBIC_KEYS_PREHASHED: return launch_map_kind<PHOBIC_KEYS_PREHASHED>(in, n, a, none, grid, st, false);
    default: return launch_map_kind<PHOBIC_KEYS_STRINGS>(in, n, a, none, grid, st, false);
    }
}

cudaError_t launch_scatter(int kind, const KeyInput &in, uint64_t n, const ScatterArgs &a, int grid, cudaStream_t st) {
    MapArgs none{};
    switch (kind) {
    case PHOBIC_KEYS_U64: return launch_map_kind<PHOBIC_KEYS_U64>(in, n, none, a, grid, st, true);
    case PHOBIC_KEYS_BYTES16: return launch_map_kind<PHOBIC_KEYS_BYTES16>(in, n, none, a, grid, st, true);
    case PHOBIC_KEYS_PREHASHED: return launch_map_kind<PHOBIC_KEYS_PREHASHED>(in, n, none, a, grid, st, true);
    default: return launch_map_kind<PHOBIC_KEYS_STRINGS>(in, n, none, a, grid, st, true);
    }
}

}  // namespace phobicb200
