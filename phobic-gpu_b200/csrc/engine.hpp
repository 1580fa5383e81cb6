// Host-side engine: device arenas, per-stream workers and the build pipeline
// that replaces BuildInvocation::run (include/phobicGpu/mphf_builder.h:225-292).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "phobic_b200.h"

namespace phobicb200 {

struct SearchShape;

// A grow-only device memory pool carved into 256-byte aligned slices; every
// slice lives until the next reset().  One arena serves one stream, so reuse
// across builds is ordered by that stream.
class DeviceArena {
  public:
    ~DeviceArena() { release(); }
    // Grows the pool to at least `bytes`; cudaErrorMemoryAllocation, without calling
    // cudaMalloc, when that exceeds the limit (if one is set).
    cudaError_t reserve(size_t bytes);
    void reset() { used_ = 0; }
    void *take(size_t bytes);
    size_t capacity() const { return cap_; }
    void release();
    // Upper bound on the pool's size; 0 = none.  A pool above a new limit is released.
    void set_limit(size_t bytes) {
        limit_ = bytes;
        if (limit_ && cap_ > limit_) release();
    }

  private:
    char *base_ = nullptr;
    size_t cap_ = 0, used_ = 0, limit_ = 0;
};

// A grow-only pinned host buffer.
class PinnedBuffer {
  public:
    ~PinnedBuffer() { release(); }
    cudaError_t reserve(size_t bytes);
    void *data() const { return p_; }
    void release();

  private:
    void *p_ = nullptr;
    size_t cap_ = 0;
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// One CUDA stream with its arena, events and pinned status/table buffers.
struct Worker {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    DeviceArena arena;
    PinnedBuffer pinned;  // set table on the way in, per-set error words on the way out
    // Results bound for pageable host memory are copied into `stage` on the stream and
    // from there to their destination by finish_sets.
    struct HostCopy {
        void *dst;
        size_t off, bytes;
    };
    PinnedBuffer stage;
    std::vector<HostCopy> pending_copies;
    // Inputs in pageable host memory go up through two pinned chunk buffers (upload()).
    PinnedBuffer up_stage;
    cudaEvent_t up_ev[2] = {};
    uint32_t pending_sets = 0;
    uint32_t pending_kernels = 0;  // kernels the last enqueued build launched
    unsigned long long *pending_err = nullptr;  // host view of the error words of the last build
    uint64_t timeout_ms = 120000;
    uint32_t search_group = 0;     // phobic_tuning::search_group (0 = automatic)
    uint32_t search_pipeline = 0;  // phobic_tuning::search_pipeline
    // The device stages of a build (memsets, K1-K4, status copy) as a CUDA graph: a build
    // whose launches are those of the previous build (same sizes, parameters, search shape
    // and buffers) is captured the second time in a row and replayed from then on.
    uint32_t graphs_off = 0;              // phobic_tuning::graphs_off
    std::vector<uint64_t> graph_key;      // launch identity of the last build
    cudaGraphExec_t graph_exec = nullptr;  // captured stages of graph_key, if any
    bool pending_graph = false;           // the last enqueued build replayed graph_exec
    void drop_graph();

    phobic_status init(int device, std::string *err);
    void destroy();
};

struct DebugOut {
    uint32_t *keys4 = nullptr;         // host [4n]
    uint32_t *bucket_sizes = nullptr;  // host [partitions * buckets]
};

// Validates parameters; fills the derived capacity and pilot-counter cap.
phobic_status check_params(const phobic_params *params, uint32_t *cap, uint32_t *k_max, std::string *err);
phobic_status check_keys(const phobic_keys *keys, std::string *err);

// Device bytes one build of these sets needs from a worker's arena.
uint64_t sets_arena_bytes(const phobic_keys *sets, uint32_t nsets, const phobic_params *params,
                          const phobic_result *results, bool debug);

// Enqueue one build of nsets key sets on the worker's stream (no wait).  All sets
// share one kind and one on_device flag; results[s] receives set s.
phobic_status enqueue_sets(Worker &w, const phobic_keys *sets, uint32_t nsets, const phobic_params *params,
                           const phobic_result *results, const DebugOut *dbg, std::string *err);

// Wait for the last enqueued build; statuses[s] (optional) gets each set's status.
// Returns the first failing set's status.
phobic_status finish_sets(Worker &w, phobic_status *statuses, phobic_timings *t, std::string *err);

// Bounded wait on an event: polls cudaEventQuery until done or timeout.
phobic_status wait_event(cudaEvent_t ev, uint64_t timeout_ms, std::string *err);
// The same bounded wait on all work queued on a stream (cudaStreamQuery).
phobic_status wait_stream(cudaStream_t s, uint64_t timeout_ms, std::string *err);
// Bound of the host-side waits: PHOBIC_TIMEOUT_MS from the environment, else 120 s.
uint64_t env_timeout_ms();

// Failure injection on the host (tests of the keys-changed guard): a one-shot request,
// set by phobic_debug_change_key, to XOR one u64 key with a mask between the counting
// pass (K1) and the placing pass (K3) of the next build of one set of device-visible
// u64 keys with more than `index` keys.  Returns true (and clears the request) when
// this build takes it.
bool take_key_change(uint64_t n, int kind, uint64_t *index, uint64_t *mask);
void set_key_change(uint64_t index, uint64_t mask);

phobic_status cuda_status(cudaError_t e, const char *what, std::string *err);

// Returns the status of a failed CUDA call from the enclosing function (which has
// a std::string *err).
#define PHB_TRY(expr, what)                                  \
    do {                                                     \
        phobic_status s_ = cuda_status((expr), (what), err); \
        if (s_ != PHOBIC_OK) return s_;                      \
    } while (0)

// Encoding of a build's result on the device (compact-vector encoders; see
// phobic_encode_gpu).  out_arena holds the packed bytes when they cannot be
// written to `out` directly.
phobic_status run_encode_gpu(Worker &w, DeviceArena &out_arena, int pilot_encoder, int offset_encoder,
                             const phobic_result *built, uint32_t partitions, const phobic_params *params,
                             uint8_t *out, size_t cap, int out_on_device, size_t *size, double *bits_per_key,
                             std::string *err);

// Query / verification over raw build output.
phobic_status run_query(Worker &w, const phobic_keys *keys, const phobic_params *params, uint32_t partitions,
                        const phobic_result *built, uint32_t *positions, uint64_t *bad, std::string *err);

// Runs the scan with a never-scheduled first tile (bounded-wait test); *observed gets
// the status the kernel recorded.
phobic_status run_stalled_wait(Worker &w, uint32_t wait_ms, phobic_status *observed, std::string *err);

// Measured integer throughput of the device for the pilot hash's mix round (shift, xor,
// multiply), all SMs at full occupancy: 32-bit operations per second and the kernel time.
phobic_status measure_int_peak(Worker &w, double *ops_per_s, double *ms, std::string *err);
// cudaFuncAttributes::binaryVersion of the library's kernels on `device` (100 = sm_100).
phobic_status kernel_binary_version(int device, int *version, std::string *err);

// Launch shape of the search for a build of `partitions` partitions: the context's
// setting, else the autotuner's table, else group 0 (launch_search's rule).
SearchShape choose_search_shape(const Worker &w, const phobic_params *params, uint32_t partitions);
// Times the search's launch shapes for a ladder of partition counts at these
// parameters and writes the fastest per size class to the tuning table at path
// (NULL or "": $PHOBIC_TUNING_FILE, else tuning.tsv beside the library's lib/).
phobic_status autotune(Worker &w, const phobic_params *params, const char *path, uint32_t *lines_written,
                       std::string *err);

// Default search bitmap capacity for a partition size (search.comp:21).
uint32_t default_max_partition(uint32_t partition_size);

}  // namespace phobicb200
