// Kernel argument blocks and launch entry points of the construction pipeline.
//
//   K1 map_count  keys -> partition counts + per-key rank        (kernels_map.cu)
//   K2 scan       partition counts -> partition offsets          (kernels_scan.cu)
//   K3 scatter    keys -> partition-contiguous (lower pair, bucket) records
//   K4 search     per partition: bucket sort + pilot search       (kernels_search.cu)
//   Q  query      keys -> slots, bijection check                  (kernels_query.cu)
#pragma once

#include "common.cuh"

namespace phobicb200 {

constexpr int kMapThreads = 256;
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;  // elements per thread: one tile = 4096 partitions
constexpr int kScanTile = kScanThreads * kScanItems;

struct KeyInput {
    const void *data;
    const uint64_t *offsets;  // strings only
};

struct MapArgs {
    uint32_t partitions;
    uint32_t buckets;
    const uint32_t *fulcs;  // [2048] device
    uint32_t *part_count;   // [partitions], zeroed
    uint32_t *rank;         // [n]
    uint4 *mapped;          // [n] {p, b, lower1, lower2}, strings only (else null)
    uint4 *debug_keys;      // [n] hashed Keys, debug builds only (else null)
    unsigned long long *err;
};

struct ScatterArgs {
    uint32_t partitions;
    const uint32_t *fulcs;
    const uint32_t *part_off;  // [partitions + 1]
    const uint32_t *rank;
    const uint4 *mapped;
    uint2 *lowers;  // [n]
    uint16_t *bkt;  // [n]
};

struct ScanArgs {
    const uint32_t *in;            // [m] partition sizes
    uint32_t *out;                 // [m + 1] exclusive prefix, out[m] = total
    uint32_t m;
    uint32_t cap;                  // largest allowed partition
    unsigned long long *tile_state; // [tiles], zeroed: (flag << 32) | value
    uint32_t *tile_counter;         // zeroed
    unsigned long long *err;
};

// One search job = one partition of one key set.
struct SearchArgs {
    const uint32_t *part_off;  // [partitions + 1] (of this set)
    const uint2 *lowers;       // partition-contiguous records (global key index)
    const uint16_t *bkt;
    uint2 *sorted;             // scratch, same indexing as lowers
    uint32_t *pilots;          // [buckets * partitions]
    uint32_t *debug_sizes;     // [partitions * buckets] or null
    uint32_t partitions;
    uint32_t buckets;
    uint32_t cap;
    uint32_t k_max;
    unsigned long long *err;
};

struct QueryArgs {
    uint32_t partitions;
    uint32_t buckets;
    const uint32_t *fulcs;
    const uint32_t *pilots;
    const uint32_t *part_off;
    uint32_t *positions;  // [n] or null
    uint32_t *seen;       // bitmap [ceil(n_built/32)] or null
    unsigned long long *bad;
    uint32_t n_built;
};

// Key of index i for each input kind (hasher.hpp:22-66).
template <int KIND>
__device__ __forceinline__ Key4 load_key(const KeyInput &in, uint64_t i) {
    if constexpr (KIND == PHOBIC_KEYS_U64) {
        uint64_t v = __ldg(static_cast<const unsigned long long *>(in.data) + i);
        return key_from_hash(xxh3::hash_u64(v));
    } else if constexpr (KIND == PHOBIC_KEYS_BYTES16) {
        const unsigned long long *r = static_cast<const unsigned long long *>(in.data) + 2 * i;
        return key_from_hash(xxh3::hash_16(__ldg(r), __ldg(r + 1)));
    } else if constexpr (KIND == PHOBIC_KEYS_PREHASHED) {
        const uint32_t *r = static_cast<const uint32_t *>(in.data) + 4 * i;
        return Key4{__ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3)};
    } else {
        uint64_t a = __ldg(reinterpret_cast<const unsigned long long *>(in.offsets) + i);
        uint64_t b = __ldg(reinterpret_cast<const unsigned long long *>(in.offsets) + i + 1);
        return key_from_hash(xxh3::hash_bytes(static_cast<const uint8_t *>(in.data) + a, (size_t)(b - a)));
    }
}

// Shared-memory bytes one warp of K4 needs for a partition capacity and bucket count.
size_t search_warp_smem(uint32_t buckets, uint32_t cap);
// Warps (= partitions in flight) per K4 CTA; 0 when one warp's state does not fit.
int search_warps_per_cta(uint32_t buckets, uint32_t cap);
constexpr int kSearchWarps = 8;
constexpr size_t kSearchSmemLimit = 227 * 1024;

cudaError_t launch_map_count(int kind, const KeyInput &in, uint64_t n, const MapArgs &a, int grid, cudaStream_t st);
cudaError_t launch_scatter(int kind, const KeyInput &in, uint64_t n, const ScatterArgs &a, int grid, cudaStream_t st);
cudaError_t launch_scan(const ScanArgs &a, cudaStream_t st);
cudaError_t launch_search(const SearchArgs &a, cudaStream_t st);
cudaError_t launch_query(int kind, const KeyInput &in, uint64_t n, const QueryArgs &a, int grid, cudaStream_t st);

}  // namespace phobicb200
