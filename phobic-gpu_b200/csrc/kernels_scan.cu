// K2: partition offsets by a single-pass decoupled-lookback exclusive scan.
//
// Replaces the multi-level prefix sum of the reference (shaders/prefix_sum.comp:18-88,
// prefix_sum_offset.comp:13-19, driven by PrefixSumStage::addCommands,
// src/prefix_sum_stage.cpp:42-86) and the host's leading zero
// (include/phobicGpu/mphf_builder.h:254-257): out[0] = 0, out[p + 1] = out[p] + size[p].
// The scanned array is the (partition, chunk) count matrix of K1, so the prefix
// is at once every partition's record offset and every chunk's scatter cursor.
// A second small kernel checks every partition against the search bitmap
// capacity, which the reference leaves unchecked (search.comp:21).
//
// Each CTA takes the next tile id from a counter, so every tile it waits on was
// started before it; the wait on a predecessor is still bounded in time
// (ScanArgs::wait_ns), after which the CTA reports PHOBIC_ERR_TIMEOUT and ends.
#include "kernels.cuh"

namespace phobicb200 {

namespace {
constexpr unsigned long long kFlagAggregate = 1ull << 32;
constexpr unsigned long long kFlagInclusive = 2ull << 32;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(kFullMask, v, d);
        if (lane >= d) v += t;
    }
    return v;
}
}  // namespace

__global__ void __launch_bounds__(kScanThreads) k_scan(ScanArgs a) {
    constexpr int kWarps = kScanThreads / 32;
    __shared__ uint32_t s_tile, s_prefix, s_total;
    __shared__ uint32_t s_warp[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if ((uint64_t)tile * kScanTile >= a.m) return;  // only when tile ids were skipped on purpose
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;

    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        uint64_t idx = base + j;
        v[j] = idx < a.m ? a.in[idx] : 0u;
        sum += v[j];
    }

    uint32_t incl = warp_incl_scan(sum, lane);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? s_warp[lane] : 0u;
        uint32_t wi = warp_incl_scan(w, lane);
        if (lane < kWarps) s_warp[lane] = wi - w;
        if (lane == kWarps - 1) s_total = wi;
    }
    __syncthreads();
    const uint32_t total = s_total;

    if (threadIdx.x == 0) {
        uint32_t prefix = 0;
        if (tile == 0) {
            atomicExch(&a.tile_state[0], kFlagInclusive | total);
        } else {
            atomicExch(&a.tile_state[tile], kFlagAggregate | total);
            int64_t j = (int64_t)tile - 1;
            const unsigned long long t0 = global_ns();
            while (j >= 0) {
                unsigned long long s = *reinterpret_cast<volatile unsigned long long *>(&a.tile_state[j]);
                unsigned long long flag = s & ~0xFFFFFFFFull;
                if (flag == 0) {
                    if (global_ns() - t0 > a.wait_ns) {
                        for (uint32_t q = 0; q < a.nsets; q++) report_error(&a.err[q], 0, PHOBIC_ERR_TIMEOUT);
                        break;
                    }
                    __nanosleep(200);
                    continue;
                }
                prefix += (uint32_t)s;
                if (flag == kFlagInclusive) break;
                j--;
            }
            atomicExch(&a.tile_state[tile], kFlagInclusive | (uint32_t)(prefix + total));
        }
        s_prefix = prefix;
    }
    __syncthreads();

    uint32_t run = s_prefix + s_warp[warp] + incl - sum;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        uint64_t idx = base + j;
        if (idx < a.m) {
            a.out[idx] = run;
            if (a.cursor) a.cursor[idx] = run;
        }
        run += v[j];
    }
    // The thread holding the last element also writes the total.
    if (base <= (uint64_t)a.m - 1 && (uint64_t)a.m - 1 < base + kScanItems) a.out[a.m] = run;
}

cudaError_t launch_scan(const ScanArgs &a, cudaStream_t st) {
    if (a.m == 0) return cudaSuccess;
    uint32_t tiles = (a.m + kScanTile - 1) / kScanTile;
    ScanArgs b = a;
    if (!b.wait_ns) b.wait_ns = kSpinTimeoutNs;
    k_scan<<<tiles, kScanThreads, 0, st>>>(b);
    return cudaGetLastError();
}

__global__ void k_check_sizes(const uint32_t *out, uint32_t M, uint32_t stride, uint32_t cap, const uint32_t *part_base,
                              uint32_t nsets, unsigned long long *err, PartArgs part, bool seed) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= M) return;
    const uint32_t start = out[(size_t)g * stride];
    if (seed) {
        part.pcur[g] = start;
        if ((g & ((1u << part.wshift) - 1)) == 0) part.bincur[g >> part.wshift] = start;
    }
    const uint32_t size = out[(size_t)(g + 1) * stride] - start;
    if (size > cap) {
        const uint32_t set = nsets == 1 ? 0u : find_set(part_base, nsets, g);
        report_error(&err[set], g - part_base[set], PHOBIC_ERR_PARTITION_OVERFLOW);
    }
}

cudaError_t launch_check_sizes(const uint32_t *out, uint32_t M, uint32_t stride, uint32_t cap,
                               const uint32_t *part_base, uint32_t nsets, unsigned long long *err,
                               const PartArgs *part, cudaStream_t st) {
    if (M == 0) return cudaSuccess;
    PartArgs p{};
    if (part) p = *part;
    k_check_sizes<<<(M + 255) / 256, 256, 0, st>>>(out, M, stride, cap, part_base, nsets, err, p, part != nullptr);
    return cudaGetLastError();
}

__global__ void k_skip_tiles(uint32_t *tile_counter, uint32_t skip) { *tile_counter = skip; }

cudaError_t launch_scan_stalled(const ScanArgs &a, uint32_t skip, cudaStream_t st) {
    if (a.m == 0) return cudaSuccess;
    uint32_t tiles = (a.m + kScanTile - 1) / kScanTile;
    k_skip_tiles<<<1, 1, 0, st>>>(a.tile_counter, skip);
    ScanArgs b = a;
    if (!b.wait_ns) b.wait_ns = kSpinTimeoutNs;
    k_scan<<<tiles, kScanThreads, 0, st>>>(b);
    return cudaGetLastError();
}

}  // namespace phobicb200
