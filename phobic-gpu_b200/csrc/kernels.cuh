// Kernel argument blocks and launch entry points of the construction pipeline.
//
//   K1 map_count  keys -> key counts per (partition, chunk)         (kernels_map.cu)
//   K2 scan       counts -> record offsets (= scatter cursors)      (kernels_scan.cu)
//                 + partition size check
//   K3 scatter    keys -> partition-contiguous (lower pair, bucket) records
//   K4 search     per partition: bucket sort + pilot search         (kernels_search.cu)
//   Q  query      keys -> slots, bijection check                    (kernels_query.cu)
//
// Every kernel works on a list of key sets.  The partitions of all sets form one
// global partition space (set s owns [part_base[s], part_base[s] + partitions));
// a plain build is a list of one set, a batched build a list of many, and the
// same launches serve both.
#pragma once

#include "common.cuh"

namespace phobicb200 {

constexpr int kMapThreads = 256;
// Chunked counting: CTA c owns the keys [c * chunk, (c + 1) * chunk) and keeps a
// counter for every partition in shared memory; the count matrix is stored
// partition-major (entry g * stride + c, stride = number of chunks), so its
// exclusive scan gives each chunk its own slot range inside every partition.
constexpr int kChunkThreads = 1024;
constexpr uint32_t kChunkCtas = 148;                 // one CTA per SM of a B200
constexpr uint64_t kChunkMinKeys = 16384;            // smallest chunk worth a CTA
constexpr uint32_t kChunkMaxPartitions = 52 * 1024;  // 32-bit shared-memory counters per CTA
// Counting only (K1): above kChunkMaxPartitions the counters are packed two to a
// 32-bit word.  A 16-bit counter that wraps is caught from the atomic's return value
// and the 65536 keys it lost are added to the chunk's count in global memory.
constexpr uint32_t kChunkNarrowMaxPartitions = 104 * 1024;
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;  // entries per thread: one tile = 4096 entries
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kSearchWarps = 8;
constexpr int kSearchCtasPerSm = 4;  // register budget: 65536 / (4 * 256) -> 64 per thread
constexpr size_t kSearchSmemLimit = 227 * 1024;

// One key set of a build.
struct SetDesc {
    const void *data;          // u64[n] | 16-byte records[n] | string bytes (device)
    const uint64_t *offsets;   // strings: [n + 1] into data (device), else null
    uint64_t key_base;         // first global key index of the set
    uint32_t n;                // keys
    uint32_t part_base;        // first global partition
    uint32_t partitions;       // ceil(n / P)
    uint32_t pad;
    uint32_t *pilots;          // [buckets * partitions] output (device)
    uint32_t *part_off;        // [partitions + 1] output (device)
};

// Set lookup: the largest s with base[s] <= x, for a table with base[nsets] = total.
template <typename T>
__device__ __forceinline__ uint32_t find_set(const T *base, uint32_t nsets, T x) {
    uint32_t lo = 0, hi = nsets;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Launch plan of K1/K3: chunked shared-memory counters when every partition's
// counter fits in one CTA's shared memory, else one global counter per partition.
struct MapPlan {
    bool chunked;
    uint32_t stride;  // count-matrix entries per partition (chunks, or 1)
    uint32_t grid;
    uint64_t chunk;   // keys per CTA (chunked plan)
    bool narrow;      // chunked with 16-bit counters: K1 counting only, launch_scatter refuses it
};
MapPlan plan_map(uint64_t total_keys, uint64_t partitions, int sm_count);

struct MapArgs {
    const SetDesc *sets;
    const uint64_t *key_base;  // [nsets + 1] global key index of each set
    uint32_t nsets;
    uint32_t buckets;
    uint64_t total_keys;
    const uint32_t *fulcs;     // [2048]
    uint32_t *counts;          // [M * stride] K1: zeroed counts;  K3: cursors (start = record offset)
    uint4 *mapped;             // strings: [total] {global partition, bucket, lower1, lower2}
    uint4 *debug_keys;         // [total] hashed Keys (debug builds) or null
    uint2 *lowers;             // K3 output [total]
    uint16_t *bkt;             // K3 output [total]
    unsigned long long *err;   // [nsets]
    uint32_t M;                // global partitions
    uint32_t stride;           // MapPlan::stride
    uint64_t chunk;            // MapPlan::chunk
};

// Two-pass partition of the records (kernels_part.cu).
constexpr int kPartThreads = 512;
constexpr int kPartItems = 8;
constexpr int kPartTile = kPartThreads * kPartItems;  // records per tile
constexpr uint32_t kMaxBins = 512;                    // coarse bins of pass 1 (upper bound)
constexpr uint32_t kTargetBins = 256;                 // coarse bins aimed for
constexpr uint32_t kLocalRange = 4096;                // partition ids one pass-2 tile may span

struct PartArgs {
    uint4 *inter;       // [total] {lower1, lower2, global partition, bucket}, coarse-bin order
    uint32_t *bincur;   // [nbins] cursors, start = offset of the bin's first partition
    uint32_t *pcur;     // [M] cursors, start = partition offset
    uint32_t wshift;    // coarse bin = partition >> wshift
    uint32_t nbins;     // ceil(M / 2^wshift) <= kMaxBins
    uint32_t M;         // partitions (records naming another are not placed)
};
// Smallest shift giving at most kTargetBins coarse bins, lowered (up to kMaxBins bins)
// until two bins span at most kLocalRange partitions.
uint32_t part_wshift(uint64_t partitions);

struct ScanArgs {
    const uint32_t *in;              // [m] count matrix, partition-major
    uint32_t *out;                   // [m + 1] exclusive prefix, out[m] = total
    uint32_t *cursor;                // [m] copy of out[0..m) (global-counter scatter cursors) or null
    uint32_t m;                      // partitions * stride
    unsigned long long *tile_state;  // [tiles], zeroed: (flag << 32) | value
    uint32_t *tile_counter;          // zeroed
    uint32_t nsets;
    unsigned long long *err;         // [nsets]
    unsigned long long wait_ns;      // bound of the look-back wait on a predecessor tile
};

struct SearchArgs {
    const SetDesc *sets;
    const uint32_t *part_base;  // [nsets + 1]
    uint32_t nsets;
    uint32_t M;                 // global partitions
    const uint32_t *G;          // [M * gstride + 1] record offsets; partition g spans [G[g*gstride], G[(g+1)*gstride])
    uint32_t gstride;
    const uint2 *lowers;        // partition-contiguous records
    const uint16_t *bkt;
    uint2 *sorted;              // scratch, same indexing as lowers
    uint32_t *debug_sizes;      // [M * buckets] or null
    uint32_t buckets;
    uint32_t cap;
    uint32_t k_max;
    uint32_t *queue;            // zeroed job counter
    unsigned long long *err;    // [nsets]
    // [M] placement cursors after K3 (or null): partition g must end at its scanned offset,
    // else its keys differed between K1 and K3.
    const uint32_t *placed = nullptr;
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

// Key i of a set, for each input kind (hasher.hpp:22-66).
template <int KIND>
__device__ __forceinline__ Key4 load_key(const void *data, const uint64_t *offsets, uint64_t i) {
    if constexpr (KIND == PHOBIC_KEYS_U64) {
        uint64_t v = __ldg(static_cast<const unsigned long long *>(data) + i);
        return key_from_hash(xxh3::hash_u64(v));
    } else if constexpr (KIND == PHOBIC_KEYS_BYTES16) {
        const unsigned long long *r = static_cast<const unsigned long long *>(data) + 2 * i;
        return key_from_hash(xxh3::hash_16(__ldg(r), __ldg(r + 1)));
    } else if constexpr (KIND == PHOBIC_KEYS_PREHASHED) {
        const uint32_t *r = static_cast<const uint32_t *>(data) + 4 * i;
        return Key4{__ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3)};
    } else {
        uint64_t a = __ldg(reinterpret_cast<const unsigned long long *>(offsets) + i);
        uint64_t b = __ldg(reinterpret_cast<const unsigned long long *>(offsets) + i + 1);
        return key_from_hash(xxh3::hash_bytes(static_cast<const uint8_t *>(data) + a, (size_t)(b - a)));
    }
}

// Shared-memory bytes one warp of K4 needs for a partition capacity and bucket count.
size_t search_warp_smem(uint32_t buckets, uint32_t cap);
// Warps (= partitions in flight) per K4 CTA; 0 when one warp's state does not fit.
int search_warps_per_cta(uint32_t buckets, uint32_t cap);

cudaError_t launch_map_count(int kind, const MapArgs &a, const MapPlan &plan, cudaStream_t st);
cudaError_t launch_scatter(int kind, const MapArgs &a, const MapPlan &plan, cudaStream_t st);
cudaError_t launch_scan(const ScanArgs &a, cudaStream_t st);
// Partition sizes out[(g+1)*stride] - out[g*stride] checked against cap (the search
// bitmap capacity); an oversized partition is reported as PHOBIC_ERR_PARTITION_OVERFLOW.
// With a PartArgs (else null) it also seeds the partition and bin cursors.
cudaError_t launch_check_sizes(const uint32_t *out, uint32_t M, uint32_t stride, uint32_t cap,
                               const uint32_t *part_base, uint32_t nsets, unsigned long long *err,
                               const PartArgs *part, cudaStream_t st);
// K3, two passes (pass 1 hashes the keys again, or reads K1's mapped records for strings).
cudaError_t launch_partition(int kind, const MapArgs &a, const PartArgs &p, int sm_count, cudaStream_t st);
// The scan with its first `skip` tile ids never handed out, so the tiles after them
// wait on predecessors that never publish: the bounded wait must end in
// PHOBIC_ERR_TIMEOUT (failure-detection tests).
cudaError_t launch_scan_stalled(const ScanArgs &a, uint32_t skip, cudaStream_t st);
// Launch shape of K4: warps that search one partition together (1, or groups of 2, 4, 8;
// 0 = chosen from the partition count by search_shape_for) and, for a group, whether it
// searches several small buckets at once (bucket pipeline) or several pilot counters of one
// bucket (k-split).
struct SearchShape {
    int group = 0;
    bool pipeline = false;
};
cudaError_t launch_search(const SearchArgs &a, int sm_count, cudaStream_t st, SearchShape shape = SearchShape{});
// Default shape when the autotuner's table has no line for a build, fitted to the B200's
// measurements: bucket pipelines of 8 warps up to 256 partitions, of 4 up to 512, of 2 up
// to 1024, else one warp per partition; a group only while the groups fit one wave of the
// group kernel.
SearchShape search_shape_for(uint32_t partitions, int sm_count);
size_t search_group_smem(uint32_t buckets, uint32_t cap, int W);
// First failed bounds check of each kernel file in the checked build (source line, 0 =
// none; always 0 in the normal build); reset clears it.
unsigned int check_line_map(bool reset);
unsigned int check_line_part(bool reset);
unsigned int check_line_search(bool reset);
// splitmix64 stream on the device: out[i] = the finalizer of seed + (i + 1) * 0x9E3779B97F4A7C15
// (synthetic keys of the autotuner).
cudaError_t launch_splitmix(uint64_t *out, uint64_t n, uint64_t seed, cudaStream_t st);
// Failure injection (tests): keys[index] ^= mask, one thread, on stream st.
cudaError_t launch_change_key(void *keys, uint64_t index, uint64_t mask, cudaStream_t st);
cudaError_t launch_query(int kind, const void *data, const uint64_t *offsets, uint64_t n, const QueryArgs &a, int grid,
                         cudaStream_t st);

}  // namespace phobicb200
