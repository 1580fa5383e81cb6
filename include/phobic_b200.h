/*
 * phobic_b200.h -- C ABI of the B200 PHOBIC minimal-perfect-hash construction engine.
 *
 * The reference (stefanfred/PHOBIC-GPU) builds an MPHF with
 *     MPHFbuilder::build(const std::vector<keyType>&, Mphf&)   include/phobicGpu/mphf_builder.h:47-48,315-321
 * which hashes the keys on the host (mphf_builder.h:201-216), runs seven Vulkan
 * compute stages (mphf_builder.h:137-199) and hands two arrays to the encoders
 * through Mphf::setData (mphf.hpp:65-75):
 *     pilots[buckets * partitions]      bucket-major, pilots[b * partitions + p]  (search.comp:170-174)
 *     partition_offsets[partitions + 1] exclusive prefix of partition sizes, [0] = 0 (mphf_builder.h:254-257)
 * This ABI replaces the host hash, the Vulkan runtime and the seven stages: it takes
 * keys and returns exactly those two arrays.  The C++ layer (phobic_gpu_mphf.hpp in the
 * package) keeps the reference's MPHFbuilder / MPHF / encoder surface on top of it.
 *
 * Conventions: plain pointers and sizes; every call returns a phobic_status; host or
 * device buffers are named by flags; a context is used by one thread at a time.
 */
#ifndef PHOBIC_B200_H
#define PHOBIC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PHOBIC_API __attribute__((visibility("default")))
#else
#define PHOBIC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PHOBIC_ABI_VERSION 1
#define PHOBIC_FULCRUMS 2048 /* shaders/constants.glsl:1 */
#define PHOBIC_MAX_BUCKET 256 /* sort_sum.comp bins: bucket sizes 1..256 */

/* Status codes.  The reference throws std::runtime_error on Vulkan errors
 * (include/app/check.h:7-25) and has undefined behaviour on overflow; here every
 * condition is a code, and the C++ layer rethrows std::runtime_error. */
typedef enum phobic_status {
    PHOBIC_OK = 0,
    PHOBIC_ERR_INVALID = 1,            /* bad argument, or a bucket id >= buckets from the fulcrum table */
    PHOBIC_ERR_OOM = 2,                /* device or pinned-host allocation failed */
    PHOBIC_ERR_BUCKET_OVERFLOW = 3,    /* a bucket of more than 256 keys */
    PHOBIC_ERR_PARTITION_OVERFLOW = 4, /* a partition above max_partition_size keys */
    PHOBIC_ERR_SEARCH_LIMIT = 5,       /* pilot counter reached its limit */
    PHOBIC_ERR_TIMEOUT = 6,            /* a bounded wait expired */
    PHOBIC_ERR_CUDA = 7,               /* CUDA runtime error (detail in phobic_last_error) */
    PHOBIC_ERR_DUPLICATE_KEY = 8,      /* two keys of one bucket hash identically */
    PHOBIC_ERR_BUDGET = 9,             /* request does not fit the server's memory budget */
    PHOBIC_ERR_BUSY = 10,              /* server queue full */
    PHOBIC_ERR_NO_DEVICE = 11,         /* no CUDA device / not sm_100 */
    PHOBIC_ERR_NOT_FOUND = 12,         /* unknown server ticket */
    PHOBIC_ERR_KEYS_CHANGED = 13       /* the build's passes read different keys: device keys were
                                          written while the build ran (order them before the call) */
} phobic_status;

/* Key kinds (hasher.hpp:22-66). */
typedef enum phobic_key_kind {
    PHOBIC_KEYS_U64 = 0,       /* uint64_t[n], hashed as 8 little-endian bytes (xxhash::hash(uint64_t)) */
    PHOBIC_KEYS_BYTES16 = 1,   /* 16-byte records hashed as 16 bytes (std::pair<u64,u64>, or Key under xxhash) */
    PHOBIC_KEYS_PREHASHED = 2, /* 16-byte Key records used as-is (nohash, hasher.hpp:22-27) */
    PHOBIC_KEYS_STRINGS = 3    /* ragged byte strings: data + offsets[n+1] (xxhash::hash(std::string)) */
} phobic_key_kind;

/* Construction parameters.  Derived on the host from MPHFconfig
 * (mphf_config.h:26-64); phobic_config() computes them. */
typedef struct phobic_params {
    uint32_t partition_size;     /* P: expected keys per partition */
    uint32_t buckets;            /* B: buckets per partition (1..65535) */
    uint32_t max_partition_size; /* search bitmap capacity; 0 = 32*floor(1.5P/32) (search.comp:21) */
    uint32_t max_pilot_counter;  /* cap on the pilot counter k; 0 = 1<<20 (also bounded by 2^31/ps) */
    uint32_t fulcrums[PHOBIC_FULCRUMS]; /* bucket mapping table (mphf_config.h:44-55) */
} phobic_params;

typedef struct phobic_keys {
    int32_t kind;            /* phobic_key_kind */
    int32_t on_device;       /* 1: data/offsets are device pointers of the context's device */
    uint64_t n;              /* number of keys (< 2^32, as mphf_builder.h:56) */
    const void *data;        /* u64[n] | 16-byte records[n] | string bytes */
    const uint64_t *offsets; /* strings only: offsets[n+1] into data */
} phobic_keys;

typedef struct phobic_result {
    int32_t on_device;           /* 1: the two arrays are device pointers */
    uint32_t *pilots;            /* [buckets * partitions], caller-allocated */
    uint32_t *partition_offsets; /* [partitions + 1], caller-allocated */
} phobic_result;

/* Stage times in milliseconds, measured with CUDA events on the build stream.
 * Labels follow the reference's HostTimer labels (mphf_builder.h:138-146, :229-290). */
typedef struct phobic_timings {
    float input_transfer;     /* host -> device copy of the keys (overlapped with bucket_sizes) */
    float bucket_sizes;       /* hash + partition count (kernel K1) */
    float partition_offsets;  /* decoupled-lookback scan (kernel K2) */
    float key_redistribution; /* partition scatter (kernel K3) */
    float search;             /* bucket sort + pilot search (kernel K4) */
    float result_transfer;    /* device -> host copy of pilots and offsets */
    float total;              /* first event to last event */
    uint32_t kernels;         /* kernels launched by the call */
    uint32_t graph_replays;   /* builds of the call whose device stages ran as one replayed
                               * CUDA graph (see phobic_tuning::graphs_off) */
} phobic_timings;

/* Launch shapes of a context's builds (no counterpart in the reference, whose shapes are
 * specialisation constants fixed per pipeline, src/search_stage.cpp:36-37). */
typedef struct phobic_tuning {
    /* Warps that search one partition together, each trying its own pilot counter per
     * step (pilots per probe): 1, 2, 4 or 8; 0 = from the autotuner's table when it holds
     * these parameters, else from the partition count. */
    uint32_t search_group;
    /* With search_group 2, 4 or 8: 1 = the group searches several small buckets at once
     * (bucket pipeline: warp w takes the w-th next bucket of at most 32 keys, results are
     * committed in order while their slots stay free), 0 = several pilot counters of one
     * bucket (k-split).  Either way the pilots are those of the sequential search. */
    uint32_t search_pipeline;
    /* 0 (default): a build of at most 2048 partitions whose launches are exactly those of the
     * context's previous build (same sizes, parameters, search shape and device buffers; keys
     * and results may hold new contents) is captured as a CUDA graph the second time in a row
     * and replayed as one graph launch from then on; the memsets, kernels, stage events and
     * status copy of the build are its nodes.  Larger builds, builds with debug outputs and
     * builds on a stream the caller is capturing launch stage by stage.  1: every build
     * launches its stages one by one. */
    uint32_t graphs_off;
    uint32_t reserved[5];
} phobic_tuning;

typedef struct phobic_ctx phobic_ctx;
typedef struct phobic_server phobic_server;

/* ------------------------------------------------------------------ setup */

/* Sets the launch shapes of the context's later builds (all zero = automatic). */
PHOBIC_API phobic_status phobic_ctx_set_tuning(phobic_ctx *ctx, const phobic_tuning *tuning);

/* No counterpart in the reference (its shapes are per-pipeline specialisation constants,
 * src/search_stage.cpp:36-37).  Autotuner: builds synthetic u64 keys (splitmix64 on the
 * device) of 16, 64, 256, 512, 768, 1024, 2048 and 4096 partitions at these parameters with
 * every search shape it knows (one warp per partition; k-split groups of 2 and 4 warps;
 * bucket pipelines of 2, 4 and 8 warps) on three key sets per size (a build of few
 * partitions lasts as long as its slowest partition, which varies with the keys), and writes
 * the shape with the lowest mean build time per size class, with every measured time, to the
 * tab-separated tuning table at path (NULL or "": $PHOBIC_TUNING_FILE, else tuning.tsv in the
 * package directory beside the library's lib/), keeping the table's lines for other devices
 * and parameters.  Builds with automatic tuning then take their shape from the table: the
 * line of their device, partition size, bucket count and partition capacity with the smallest
 * size class that holds their partition count.  *lines_written (optional) = size classes
 * written. */
PHOBIC_API phobic_status phobic_autotune(phobic_ctx *ctx, const phobic_params *params, const char *path,
                                         uint32_t *lines_written);

/* Human-readable name of a status code. */
PHOBIC_API const char *phobic_status_string(phobic_status s);

/* Number of partitions for n keys: ceil(n / P) (mphf_builder.h:90). */
PHOBIC_API uint32_t phobic_partitions(uint64_t n, uint32_t partition_size);

/* MPHFconfig arithmetic (mphf_config.h:26-64, bucketers.h:20-50):
 * bucketer 0 = OptBucketer (the default), 1 = UniformBucketer, 2 = SkewBucketer;
 * bucketer_ctor != 0 selects MPHFconfig(Bucketer*, λ, P), which rounds P/λ instead of
 * taking its ceiling.  Fills every field of *out (max_pilot_counter = 0). */
PHOBIC_API phobic_status phobic_config(double lambda, uint32_t partition_size, int bucketer, int bucketer_ctor,
                            phobic_params *out);

/* Create a context on a CUDA device (one stream, pooled device buffers). */
PHOBIC_API phobic_status phobic_ctx_create(int device, phobic_ctx **out);
PHOBIC_API phobic_status phobic_ctx_destroy(phobic_ctx *ctx);
/* Detail text of the last error on this context (never NULL). */
PHOBIC_API const char *phobic_last_error(const phobic_ctx *ctx);
/* Device bytes the context's pools hold now. */
PHOBIC_API uint64_t phobic_ctx_device_bytes(const phobic_ctx *ctx);
/* Caps the device memory of the context's build pool (0 = no cap).  A build whose
 * pool would exceed the cap fails with PHOBIC_ERR_OOM before any allocation is
 * attempted, and the context stays usable; a pool already above the cap is freed.
 * The reference allocates per build without a limit (memory.cpp:40-90). */
PHOBIC_API phobic_status phobic_ctx_set_memory_limit(phobic_ctx *ctx, uint64_t bytes);
/* The context's CUDA stream (a cudaStream_t): every kernel of its builds runs on it, so
 * callers can order their own work and time builds with events on this stream. */
PHOBIC_API void *phobic_ctx_stream(const phobic_ctx *ctx);
/* Device bytes one build of n keys needs (keys staging excluded when on_device). */
PHOBIC_API uint64_t phobic_build_bytes_needed(const phobic_keys *keys, const phobic_params *params);

/* ------------------------------------------------------------------ build
 * Replaces BuildInvocation::run (mphf_builder.h:225-292) up to, not including,
 * Mphf::setData.  Synchronous: returns when the result arrays are written. */
PHOBIC_API phobic_status phobic_build(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                           const phobic_result *result, phobic_timings *timings);

/* Convenience forms with host buffers (the reference's std::vector inputs). */
PHOBIC_API phobic_status phobic_build_u64(phobic_ctx *ctx, const uint64_t *keys, uint64_t n, const phobic_params *params,
                               uint32_t *pilots, uint32_t *partition_offsets, phobic_timings *timings);
PHOBIC_API phobic_status phobic_build_strings(phobic_ctx *ctx, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                                   const phobic_params *params, uint32_t *pilots, uint32_t *partition_offsets,
                                   phobic_timings *timings);

/* ------------------------------------------------------------------ batch
 * Many independent key sets built with one launch per stage: the partitions
 * of all sets form one work list that the search kernel's CTAs share.
 * results[i] receives set i; statuses[i] its status.  Returns the first error. */
PHOBIC_API phobic_status phobic_build_batch(phobic_ctx *ctx, const phobic_keys *sets, uint32_t nsets,
                                 const phobic_params *params, const phobic_result *results,
                                 phobic_status *statuses, phobic_timings *timings);

/* No counterpart in the reference (it has no bounded device waits to test).
 * Failure-detection hook: runs the partition-offset scan with its first tile never
 * scheduled, so the next tile's look-back waits on a flag that nothing sets.  The
 * kernel's bounded wait (wait_ms) must give up and record PHOBIC_ERR_TIMEOUT, which is
 * returned in *observed; the context stays usable afterwards. */
/* The bounds checks of the checked library (libphobic_b200_checked.so, built with
 * -DPHOBIC_CHECKED): *compiled = 1 there, 0 in the normal library.  lines[0..2] = the
 * source line of the first failed check in the key-mapping, partition and search
 * kernels (0 = none failed).  A failed check skips its memory access instead of
 * trapping.  reset != 0 clears the records.  Stands in for a memory checker, which is
 * not available on every machine (it has no counterpart in the reference, which
 * relies on Vulkan validation layers, src/app/app.cpp:96-108). */
PHOBIC_API phobic_status phobic_debug_checks(phobic_ctx *ctx, int *compiled, uint32_t *lines, int reset);
PHOBIC_API phobic_status phobic_debug_stalled_wait(phobic_ctx *ctx, uint32_t wait_ms, phobic_status *observed);

/* No counterpart in the reference.  Failure injection on the host for the guard against
 * keys that change during a build: the next build (phobic_build of one set, or
 * phobic_build_noalloc) of device-visible u64 keys with more than `index` keys runs a
 * one-thread kernel between its counting pass and its placing pass that does
 * keys[index] ^= xor_mask on the keys it builds from (the caller's device array, or the
 * context's staged copy of host keys).  The two passes then disagree and the build must
 * return PHOBIC_ERR_KEYS_CHANGED.  One shot, process-wide; xor_mask = 0 disarms it. */
PHOBIC_API phobic_status phobic_debug_change_key(uint64_t index, uint64_t xor_mask);

/* No counterpart in the reference.  Measurement: the integer throughput of the context's
 * device for the pilot hash's mixing round (x = ((x >> 16) ^ x) * 0x45d9f3b, three 32-bit
 * operations, hashing.glsl:11-17), many independent chains per thread, every SM at full
 * occupancy.  *ops_per_s = 32-bit integer operations per second (the denominator of the
 * search kernel's integer-op roofline), *kernel_ms = the timed kernel's duration. */
PHOBIC_API phobic_status phobic_measure_int_peak(phobic_ctx *ctx, double *ops_per_s, double *kernel_ms);

/* No counterpart in the reference.  cudaFuncAttributes::binaryVersion of the library's
 * kernels on the context's device: 100 for code compiled for sm_100a. */
PHOBIC_API phobic_status phobic_ctx_kernel_arch(phobic_ctx *ctx, int *binary_version);

/* ------------------------------------------------------------------ encoding
 * Mphf::setData (mphf.hpp:65-75) on the host: encodes a build's pilots and
 * partition offsets with the reference's encoders (same bytes as the reference)
 * and serialises them in visit() order: the pilot encoder, then the partition-
 * offset encoder; vectors as a size_t count followed by their elements.
 * pilot_encoder: 0 interleaved<compact>, 1 interleaved<dictionary>, 2 interleaved<rice>,
 * 3 mono<compact>, 4 mono<dictionary>, 5 interleaved_dual<rice,compact> (tradeoff),
 * 6 interleaved<elias_fano>, 7 interleaved<sdc>, 8 mono<rice>.
 * offset_encoder: 0 diff_partition<compact>, 1 direct_partition<compact>.
 * Writes at most cap bytes to out (out may be NULL); *size = the full byte count. */
PHOBIC_API phobic_status phobic_encode(int pilot_encoder, int offset_encoder, const uint32_t *pilots,
                                       const uint32_t *partition_offsets, uint32_t partitions,
                                       const phobic_params *params, float tradeoff, uint8_t *out, size_t cap,
                                       size_t *size, double *bits_per_key);

/* Mphf::setData on the GPU for the encoders made of compact vectors: pilot_encoder
 * 0 (interleaved<compact>) or 3 (mono<compact>), offset_encoder 0 (diff_partition
 * <compact>) or 1 (direct_partition<compact>); other encoders are PHOBIC_ERR_INVALID
 * (use phobic_encode).  Same bytes, in the same visit order, and the same
 * bits_per_key as phobic_encode for these encoders (interleaved_encoder.hpp:8-15,
 * mono_encoders.hpp, linear_diff_encoder.hpp:15-28, compact_vector.hpp).
 * built's arrays are read on the device when built->on_device, else copied in.
 * out (host memory, or device memory when out_on_device) receives at most cap
 * bytes and may be NULL; *size = the full byte count.  Synchronous. */
PHOBIC_API phobic_status phobic_encode_gpu(phobic_ctx *ctx, int pilot_encoder, int offset_encoder,
                                           const phobic_result *built, uint32_t partitions,
                                           const phobic_params *params, uint8_t *out, size_t cap,
                                           int out_on_device, size_t *size, double *bits_per_key);

/* Device arrays owned by the context for one build result of `partitions`
 * partitions (pilots [buckets * partitions], offsets [partitions + 1]), so that a
 * caller without its own device memory can build into the device and encode from
 * there (phobic_build with *out, then phobic_encode_gpu).  *out->on_device = 1.
 * The arrays stay valid until the next call of this function on the context or
 * its destruction. */
PHOBIC_API phobic_status phobic_ctx_result(phobic_ctx *ctx, uint32_t buckets, uint32_t partitions,
                                           phobic_result *out);

/* ------------------------------------------------------------------ query
 * MPHF::operator() (mphf.hpp:77-86) over the raw (unencoded) result arrays.
 * positions[i] = slot of key i in [0, n_built).  Arrays may live on the host
 * or the device (flags); positions follow keys->on_device. */
PHOBIC_API phobic_status phobic_query(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                           uint32_t partitions, const phobic_result *built, uint32_t *positions);

/* Bijection check (example.cpp:43-59) on the device: *bad = number of keys whose
 * slot is out of range or already taken. */
PHOBIC_API phobic_status phobic_verify(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                            const phobic_result *built, uint64_t *bad);

/* ------------------------------------------------------------------ debug
 * Intermediates of one build for parity tests (host buffers, NULL to skip):
 * keys4[4n] hashed Keys; bucket_sizes[partitions*buckets] (p-major). */
PHOBIC_API phobic_status phobic_debug_build(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                                 const phobic_result *result, uint32_t *keys4, uint32_t *bucket_sizes);

/* ------------------------------------------------------------------ no allocation
 * phobic_build_noalloc has no counterpart in the reference.  It is the plain build
 * for callers that cannot allocate device memory: a host framework that owns the
 * whole device memory pool and only hands out buffers it sized itself, a latency-
 * critical path that cannot pay cudaMalloc's implicit synchronisation, or a plugin
 * host that forbids allocation inside its callbacks.  It allocates nothing (no
 * cudaMalloc, cudaFree, pinned memory, stream or event creation); every scratch byte
 * comes from one static device array of about 20 MiB that each GPU loading this
 * library holds until the process exits.
 *   - keys: device-resident, kind U64, BYTES16 or PREHASHED, at most 1,048,576 keys
 *     in at most 65,536 partitions; larger builds return PHOBIC_ERR_BUDGET, other
 *     unsupported inputs PHOBIC_ERR_INVALID.
 *   - result: device arrays (on_device = 1), as for phobic_build.
 *   - stream: the cudaStream_t to run on (NULL = legacy default stream).  The call is
 *     synchronous: it returns after that stream has drained (waiting at most
 *     PHOBIC_TIMEOUT_MS, default 120 s), with the build's status.  It must not be made
 *     while the stream is being captured into a CUDA graph (PHOBIC_ERR_INVALID).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) for that device.  All calls share the array and it keeps
 * the last call's contents (the call clears what must start at zero).  Calls whose
 * work would overlap on the GPU would race on the array: while one call's work is
 * queued or running on a device, other calls on that device return PHOBIC_ERR_BUSY.
 * After PHOBIC_ERR_TIMEOUT the build's work is still queued on the stream and keeps
 * the array: later calls on that device return PHOBIC_ERR_BUSY until it has drained,
 * and the caller must synchronise the stream before it frees or rewrites the keys or
 * the result arrays. */
PHOBIC_API phobic_status phobic_build_noalloc(const phobic_keys *keys, const phobic_params *params,
                                              const phobic_result *result, void *stream);

/* ------------------------------------------------------------------ serving
 * A build server: a request loop that admits key sets as they arrive against a
 * device-memory budget, keeps buffers resident, overlaps admitted requests on
 * several streams, and records per-request latency. */
typedef struct phobic_server_config {
    int32_t device;
    uint32_t streams;        /* concurrent builds in flight (>= 1) */
    uint32_t queue_capacity; /* pending requests before submit returns PHOBIC_ERR_BUSY */
    uint32_t max_batch_sets; /* requests built together in one batch; 0 = no limit, 1 = one at a time */
    uint64_t budget_bytes;   /* device memory the admitted builds may hold together */
} phobic_server_config;

typedef struct phobic_server_stats {
    uint64_t completed;
    uint64_t failed;
    uint64_t keys;
    double p50_ms, p99_ms, max_ms; /* submit-to-completion latency */
    double busy_ms;                /* wall time with at least one request in flight */
    uint64_t peak_bytes;           /* largest admitted device footprint */
    uint32_t max_batch_requests;   /* most requests built together in one batch */
    uint32_t max_batches_in_flight;/* most batches queued or running on the device at once */
    uint32_t max_device_overlap;   /* most batches whose device work (first to last event on
                                      their streams) overlapped in time */
    uint32_t pad;
} phobic_server_stats;

PHOBIC_API phobic_status phobic_server_create(const phobic_server_config *cfg, phobic_server **out);
/* Copies nothing: keys and result buffers must stay valid until the request completes. */
PHOBIC_API phobic_status phobic_server_submit(phobic_server *srv, const phobic_keys *keys, const phobic_params *params,
                                   const phobic_result *result, uint64_t *ticket);
/* *done = 1 and *status set once the request finished. */
PHOBIC_API phobic_status phobic_server_poll(phobic_server *srv, uint64_t ticket, int *done, phobic_status *status);
/* Waits at most timeout_ms for the request (PHOBIC_ERR_TIMEOUT otherwise). */
PHOBIC_API phobic_status phobic_server_wait(phobic_server *srv, uint64_t ticket, uint32_t timeout_ms, phobic_status *status);
PHOBIC_API phobic_status phobic_server_drain(phobic_server *srv, uint32_t timeout_ms);
/* Sizes every stream's device arena to device_bytes and its pinned result stage to
 * pinned_bytes now, so that requests up to that size allocate nothing while the
 * streams serve (growing an arena mid-stream frees and reallocates it, which waits
 * for the whole device).  device_bytes comes from phobic_build_bytes_needed; the
 * stage holds a batch's results bound for pageable host memory.  PHOBIC_ERR_BUDGET
 * when streams x device_bytes exceeds the budget, PHOBIC_ERR_BUSY while requests
 * are pending or in flight. */
PHOBIC_API phobic_status phobic_server_reserve(phobic_server *srv, uint64_t device_bytes, uint64_t pinned_bytes);
PHOBIC_API phobic_status phobic_server_stats_get(phobic_server *srv, phobic_server_stats *out);
PHOBIC_API phobic_status phobic_server_destroy(phobic_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* PHOBIC_B200_H */
