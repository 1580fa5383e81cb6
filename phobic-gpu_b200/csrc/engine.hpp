// Host-side engine: device arenas, per-stream workers and the build pipeline
// that replaces BuildInvocation::run (include/phobicGpu/mphf_builder.h:225-292).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "phobic_b200.h"

namespace phobicb200 {

// A grow-only device memory pool carved into 256-byte aligned slices; every
// slice lives until the next reset().  One arena serves one stream, so reuse
// across builds is ordered by the stream.
class DeviceArena {
  public:
    ~DeviceArena() { release(); }
    cudaError_t reserve(size_t bytes);
    void reset() { used_ = 0; }
    void *take(size_t bytes);
    size_t capacity() const { return cap_; }
    void release();

  private:
    char *base_ = nullptr;
    size_t cap_ = 0, used_ = 0;
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// One CUDA stream with its arena, events and a pinned status word.
struct Worker {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    DeviceArena arena;
    unsigned long long *pinned_err = nullptr;  // host-pinned copy of the device error word
    uint64_t timeout_ms = 120000;

    phobic_status init(int device, std::string *err);
    void destroy();
};

struct DebugOut {
    uint32_t *keys4 = nullptr;         // host [4n]
    uint32_t *bucket_sizes = nullptr;  // host [partitions * buckets]
};

// Validates arguments; fills the derived capacity and pilot cap.
phobic_status check_build_args(const phobic_keys *keys, const phobic_params *params, uint32_t *cap,
                               uint32_t *k_max, std::string *err);

// Device bytes one build needs from a worker's arena.
uint64_t build_arena_bytes(const phobic_keys *keys, const phobic_params *params, const phobic_result *result,
                           bool debug);

// Enqueue one whole build on the worker's stream (no wait).
phobic_status enqueue_build(Worker &w, const phobic_keys *keys, const phobic_params *params,
                            const phobic_result *result, const DebugOut *dbg, std::string *err);

// Wait for the last enqueued build, decode its status and fill timings.
phobic_status finish_build(Worker &w, phobic_timings *t, std::string *err);

// Bounded wait on an event: polls cudaEventQuery until done or timeout.
phobic_status wait_event(cudaEvent_t ev, uint64_t timeout_ms, std::string *err);

phobic_status cuda_status(cudaError_t e, const char *what, std::string *err);

// Query / verification over raw build output.
phobic_status run_query(Worker &w, const phobic_keys *keys, const phobic_params *params, uint32_t partitions,
                        const phobic_result *built, uint32_t *positions, uint64_t *bad, std::string *err);

// Default search bitmap capacity for a partition size (search.comp:21).
uint32_t default_max_partition(uint32_t partition_size);

}  // namespace phobicb200
