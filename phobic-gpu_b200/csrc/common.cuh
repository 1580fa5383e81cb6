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

// Lets `func` take up to the device's opt-in shared memory per block (less its static
// shared memory) as dynamic shared memory, and checks that `bytes` fit.  The limit is a
// property of the function shared by all host threads: every caller sets this same
// value, so a launch from one thread cannot lower it under another thread's launch.
template <typename F>
inline cudaError_t allow_dynamic_smem(F *func, size_t bytes) {
    int dev = 0, optin = 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, func);
    if (e != cudaSuccess) return e;
    const int limit = optin - (int)fa.sharedSizeBytes;
    if (limit < 0 || bytes > (size_t)limit) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
}

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

// Bounds checks of the checked build (-DPHOBIC_CHECKED).  PHB_CHECK(cond) guards one
// shared- or global-memory access: in the checked build a false condition records
// the check's source line in this translation unit's status word (the first failure
// is kept) and the access is skipped; in the normal build it is `true` and compiles
// away.  Nothing traps: the kernel runs on and the host reads the word afterwards.
#ifdef PHOBIC_CHECKED
static __device__ unsigned int g_check_line;
__device__ __forceinline__ bool phb_check(bool ok, unsigned int line) {
    if (!ok) atomicCAS(&g_check_line, 0u, line);
    return ok;
}
#define PHB_CHECK(cond) ::phobicb200::phb_check((cond), __LINE__)
// This translation unit's status word (0 = no failed check); reset clears it.
static inline unsigned int read_check_line(bool reset) {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_check_line, sizeof(v)) != cudaSuccess) return 0xFFFFFFFFu;
    if (reset) {
        const unsigned int z = 0;
        cudaMemcpyToSymbol(g_check_line, &z, sizeof(z));
    }
    return v;
}
#else
#define PHB_CHECK(cond) true
static inline unsigned int read_check_line(bool) { return 0; }
#endif

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace phobicb200
