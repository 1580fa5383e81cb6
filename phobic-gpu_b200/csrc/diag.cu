// Diagnostics for measurement and tests (no counterpart in the reference):
//
//   * the measured integer peak of this GPU for the pilot hash's instruction mix,
//     the denominator of the search kernel's integer-op roofline;
//   * the architecture the library's kernels were compiled for, read through the
//     runtime (cudaFuncGetAttributes).
#include "engine.hpp"
#include "kernels.cuh"

namespace phobicb200 {
namespace {

constexpr int kPeakChains = 8;        // independent dependency chains per thread
constexpr int kPeakThreads = 256;
constexpr int kPeakOpsPerStep = 3;    // shift, xor, multiply: one mix round of the pilot hash

// Each thread runs kPeakChains independent chains of x = ((x >> 16) ^ x) * 0x45d9f3b, the
// round of the pilot hash's mixer (hashing.glsl:11-17); every round is three 32-bit
// integer operations.  The result is written only in a case that never happens for the
// seeds used, so the chains stay live without a store per thread.
__global__ void __launch_bounds__(kPeakThreads) k_int_peak(uint32_t iters, uint32_t seed, uint32_t *sink) {
    uint32_t x[kPeakChains];
#pragma unroll
    for (int i = 0; i < kPeakChains; i++) x[i] = seed ^ (threadIdx.x * 0x9E3779B9u + blockIdx.x * 0x85EBCA6Bu + i);
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < kPeakChains; i++) x[i] = ((x[i] >> 16) ^ x[i]) * 0x45d9f3bu;
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < kPeakChains; i++) r ^= x[i];
    if (r == 0x2545F491u && seed == 0xFFFFFFFFu) sink[0] = r;
}

__global__ void k_splitmix(unsigned long long *out, uint64_t n, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        out[i] = z ^ (z >> 31);
    }
}

}  // namespace

cudaError_t launch_splitmix(uint64_t *out, uint64_t n, uint64_t seed, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148 * 16);
    k_splitmix<<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<unsigned long long *>(out), n, seed);
    return cudaGetLastError();
}

phobic_status measure_int_peak(Worker &w, double *ops_per_s, double *ms, std::string *err) {
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    int per_sm = 0;
    PHB_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_int_peak, kPeakThreads, 0), "occupancy");
    const int grid = w.sm_count * (per_sm > 0 ? per_sm : 1);
    const uint32_t iters = 16384;
    w.arena.reset();
    PHB_TRY(w.arena.reserve(256), "device arena");
    uint32_t *sink = static_cast<uint32_t *>(w.arena.take(4));
    k_int_peak<<<grid, kPeakThreads, 0, w.stream>>>(64, 1u, sink);  // warm-up
    PHB_TRY(cudaGetLastError(), "int peak launch");
    float best = 0.f;
    for (int rep = 0; rep < 3; rep++) {
        PHB_TRY(cudaEventRecord(w.ev[0], w.stream), "event");
        k_int_peak<<<grid, kPeakThreads, 0, w.stream>>>(iters, 2u + rep, sink);
        PHB_TRY(cudaGetLastError(), "int peak launch");
        PHB_TRY(cudaEventRecord(w.ev[1], w.stream), "event");
        phobic_status st = wait_event(w.ev[1], w.timeout_ms, err);
        if (st != PHOBIC_OK) return st;
        float t = 0.f;
        PHB_TRY(cudaEventElapsedTime(&t, w.ev[0], w.ev[1]), "event time");
        if (rep == 0 || t < best) best = t;
    }
    const double ops = (double)grid * kPeakThreads * kPeakChains * kPeakOpsPerStep * iters;
    *ms = best;
    *ops_per_s = best > 0.f ? ops / (best * 1e-3) : 0.0;
    return PHOBIC_OK;
}

phobic_status kernel_binary_version(int device, int *version, std::string *err) {
    PHB_TRY(cudaSetDevice(device), "cudaSetDevice");
    cudaFuncAttributes fa;
    PHB_TRY(cudaFuncGetAttributes(&fa, k_int_peak), "cudaFuncGetAttributes");
    *version = fa.binaryVersion;
    return PHOBIC_OK;
}

}  // namespace phobicb200
