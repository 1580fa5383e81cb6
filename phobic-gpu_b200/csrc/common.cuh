// Shared device-side definitions for the construction kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../cpp/phobicB200/keyhash.hpp"
#include "phobic_b200.h"

namespace phobicb200 {

constexpr uint32_t kFullMask = 0xFFFFFFFFu;
constexpr uint32_t kMaxBucket = 256;         // sort_sum.comp bins cover sizes 1..256
constexpr uint32_t kDupCheckAt = 256;        // pilot counter at which a bucket is checked for duplicate keys
constexpr uint32_t kDefaultMaxPilot = 1u << 20;
constexpr unsigned long long kNoError = ~0ull;
constexpr unsigned long long kSpinTimeoutNs = 1000000000ull;  // default bound of every spin-wait: 1 s

// Nanosecond clock shared by all SMs, for time-bounded waits.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Error word: the smallest (partition << 32 | code) wins, so the reported error is
// the one of the lowest partition, and errors found before the search (code INVALID
// from the mapping, reported at partition 0) take precedence.
__device__ __forceinline__ void report_error(unsigned long long *err, uint32_t partition, uint32_t code) {
    atomicMin(err, ((unsigned long long)partition << 32) | code);
}

__device__ __forceinline__ bool fatal_before_search(unsigned long long e) {
    uint32_t code = (uint32_t)e;
    return e != kNoError && (code == PHOBIC_ERR_INVALID || code == PHOBIC_ERR_PARTITION_OVERFLOW ||
                             code == PHOBIC_ERR_TIMEOUT);
}

// a mod d for any 32-bit a and 1 <= d, with m = 0xFFFFFFFF / d precomputed:
// q = mulhi(a, m) is floor(a/d) or one less, so one correction step suffices.
struct FastMod {
    uint32_t d, m;
    __host__ __device__ static FastMod make(uint32_t d) { return FastMod{d, 0xFFFFFFFFu / d}; }
    __device__ __forceinline__ uint32_t mod(uint32_t a) const {
        uint32_t r = a - __umulhi(a, m) * d;
        return r >= d ? r - d : r;
    }
    __device__ __forceinline__ uint32_t div(uint32_t a) const {
        uint32_t q = __umulhi(a, m);
        return (a - q * d) >= d ? q + 1 : q;
    }
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace phobicb200
