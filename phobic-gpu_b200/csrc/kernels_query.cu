// Q: batched MPHF query over the raw (unencoded) build output, and the
// bijection check built on it.
//
// Query follows MPHF::operator() (include/phobicGpu/mphf.hpp:77-86): hash,
// partition = hi32(partitioner * partitions), bucket by the 64-bit fulcrum
// interpolation (mphf.hpp:42-49), pilot = pilots[bucket * partitions + p],
// slot = offset[p] + ((hash(lower1, hash(lower2, pilot / ps)) >> 1) + pilot) mod ps
// (mphf.hpp:32-40).  The bijection check is the one of example.cpp:43-59:
// every slot in range and taken once.
#include "kernels.cuh"

namespace phobicb200 {

template <int KIND>
__global__ void __launch_bounds__(kMapThreads) k_query(const void *data, const uint64_t *offsets, uint64_t n,
                                                      QueryArgs a) {
    __shared__ uint32_t sf[kFulcrums];
    for (uint32_t i = threadIdx.x; i < kFulcrums; i += blockDim.x) sf[i] = a.fulcs[i];
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long bad = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Key4 k = load_key<KIND>(data, offsets, i);
        uint32_t p = partition_of(k.partitioner, a.partitions);
        uint64_t b = bucket_of_query(k.bucketer, sf);
        uint32_t pos = 0xFFFFFFFFu;
        if (b < a.buckets && p < a.partitions) {
            uint32_t pilot = a.pilots[b * a.partitions + p];
            uint32_t off = a.part_off[p], ps = a.part_off[p + 1] - off;
            if (ps) {
                FastMod fm = FastMod::make(ps);
                uint32_t kk = ps > 1 ? fm.div(pilot) : 0u;
                pos = off + fm.mod(pilot_hash(k.lower1, k.lower2, kk) + pilot);
            }
        }
        if (a.positions) a.positions[i] = pos;
        if (a.seen) {
            if (pos >= a.n_built) {
                bad++;
            } else {
                uint32_t bit = 1u << (pos & 31);
                if (atomicOr(&a.seen[pos >> 5], bit) & bit) bad++;
            }
        }
    }
    if (a.bad && bad) atomicAdd(a.bad, bad);
}

cudaError_t launch_query(int kind, const void *data, const uint64_t *offsets, uint64_t n, const QueryArgs &a, int grid,
                         cudaStream_t st) {
    switch (kind) {
    case PHOBIC_KEYS_U64: k_query<PHOBIC_KEYS_U64><<<grid, kMapThreads, 0, st>>>(data, offsets, n, a); break;
    case PHOBIC_KEYS_BYTES16: k_query<PHOBIC_KEYS_BYTES16><<<grid, kMapThreads, 0, st>>>(data, offsets, n, a); break;
    case PHOBIC_KEYS_PREHASHED: k_query<PHOBIC_KEYS_PREHASHED><<<grid, kMapThreads, 0, st>>>(data, offsets, n, a); break;
    default: k_query<PHOBIC_KEYS_STRINGS><<<grid, kMapThreads, 0, st>>>(data, offsets, n, a); break;
    }
    return cudaGetLastError();
}

}  // namespace phobicb200
