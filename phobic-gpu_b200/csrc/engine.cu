// Build pipeline on one stream: the CUDA replacement of BuildInvocation::run
// (include/phobicGpu/mphf_builder.h:225-292).
//
//   reference stage (mphf_builder.h)           here
//   initialHash (host, :201-216)          ->  K1 map_count (device XXH3)
//   input_transfer (:233-238)             ->  H2D of the raw keys (16 B Key not materialised)
//   bucket_sizes (:153-159)               ->  K1
//   bucket_sorting (:162-167)             ->  K4 (shared memory, per partition)
//   partition_offsets (:169-174)          ->  K2 decoupled-lookback scan
//   apply_partition_offsets (:176-180)    ->  K3 (offset added while scattering)
//   key_redistribution (:182-187)         ->  K3 + K4
//   search (:189-194)                     ->  K4
//   result_transfer (:196-261)            ->  D2H of pilots and offsets
#include "engine.hpp"

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "kernels.cuh"

namespace phobicb200 {

// ------------------------------------------------------------------ arena

cudaError_t DeviceArena::reserve(size_t bytes) {
    if (bytes <= cap_) return cudaSuccess;
    release();
    size_t want = align256(bytes);
    cudaError_t e = cudaMalloc(&base_, want);
    if (e != cudaSuccess) {
        base_ = nullptr;
        cudaGetLastError();
        return e;
    }
    cap_ = want;
    used_ = 0;
    return cudaSuccess;
}

void DeviceArena::release() {
    if (base_) cudaFree(base_);
    base_ = nullptr;
    cap_ = used_ = 0;
}

void *DeviceArena::take(size_t bytes) {
    size_t b = align256(bytes ? bytes : 1);
    if (used_ + b > cap_) return nullptr;
    void *p = base_ + used_;
    used_ += b;
    return p;
}

// ------------------------------------------------------------------ helpers

phobic_status cuda_status(cudaError_t e, const char *what, std::string *err) {
    if (e == cudaSuccess) return PHOBIC_OK;
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return PHOBIC_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return PHOBIC_ERR_NO_DEVICE;
    return PHOBIC_ERR_CUDA;
}

#define PHB_TRY(expr, what)                                        \
    do {                                                           \
        phobic_status s_ = cuda_status((expr), (what), err);       \
        if (s_ != PHOBIC_OK) return s_;                            \
    } while (0)

phobic_status wait_event(cudaEvent_t ev, uint64_t timeout_ms, std::string *err) {
    auto t0 = std::chrono::steady_clock::now();
    uint32_t polls = 0;
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return PHOBIC_OK;
        if (e != cudaErrorNotReady) return cuda_status(e, "device work failed", err);
        auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
        if ((uint64_t)ms > timeout_ms) {
            if (err) *err = "device work did not finish within " + std::to_string(timeout_ms) + " ms";
            return PHOBIC_ERR_TIMEOUT;
        }
        if (++polls < 2000) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

uint32_t default_max_partition(uint32_t P) {
    uint32_t words = (P + P / 2) / 32;  // mphf_config.h:61-64 / 32 bits (search.comp:21)
    return 32 * (words ? words : 1);
}

phobic_status Worker::init(int dev, std::string *err) {
    device = dev;
    PHB_TRY(cudaSetDevice(dev), "cudaSetDevice");
    int major = 0;
    PHB_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "device query");
    if (major < 10) {
        if (err) *err = "device is not sm_100 class (compute capability major " + std::to_string(major) + ")";
        return PHOBIC_ERR_NO_DEVICE;
    }
    PHB_TRY(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev), "device query");
    PHB_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto &e : ev) PHB_TRY(cudaEventCreate(&e), "cudaEventCreate");
    PHB_TRY(cudaMallocHost(&pinned_err, sizeof(unsigned long long)), "cudaMallocHost");
    if (const char *t = std::getenv("PHOBIC_TIMEOUT_MS")) timeout_ms = std::strtoull(t, nullptr, 10);
    return PHOBIC_OK;
}

void Worker::destroy() {
    if (stream) {
        cudaSetDevice(device);
        if (ev[7] && cudaEventRecord(ev[7], stream) == cudaSuccess) wait_event(ev[7], timeout_ms, nullptr);
    }
    arena.release();
    for (auto &e : ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (stream) cudaStreamDestroy(stream), stream = nullptr;
    if (pinned_err) cudaFreeHost(pinned_err), pinned_err = nullptr;
}

// ------------------------------------------------------------------ sizes

static uint64_t key_bytes(const phobic_keys *k) {
    switch (k->kind) {
    case PHOBIC_KEYS_U64: return 8 * k->n;
    case PHOBIC_KEYS_BYTES16:
    case PHOBIC_KEYS_PREHASHED: return 16 * k->n;
    default: return 0;
    }
}

phobic_status check_build_args(const phobic_keys *keys, const phobic_params *params, uint32_t *cap, uint32_t *k_max,
                               std::string *err) {
    auto bad = [&](const char *m) {
        if (err) *err = m;
        return PHOBIC_ERR_INVALID;
    };
    if (!keys || !params) return bad("null keys or params");
    if (keys->kind < PHOBIC_KEYS_U64 || keys->kind > PHOBIC_KEYS_STRINGS) return bad("unknown key kind");
    if (keys->n > 0xFFFFFFFFull) return bad("more than 2^32-1 keys (the reference's uint32 size, mphf_builder.h:56)");
    if (keys->n && !keys->data) return bad("null key data");
    if (keys->kind == PHOBIC_KEYS_STRINGS && keys->n && !keys->offsets) return bad("strings need offsets");
    if (params->partition_size == 0) return bad("partition_size must be > 0");
    if (params->buckets == 0 || params->buckets > 65535) return bad("buckets must be in 1..65535");
    if (params->fulcrums[kFulcrums - 1] != (params->buckets << 16))
        return bad("fulcrum table does not end at buckets << 16 (mphf_config.h:54)");
    *cap = params->max_partition_size ? params->max_partition_size : default_max_partition(params->partition_size);
    *k_max = params->max_pilot_counter ? params->max_pilot_counter : kDefaultMaxPilot;
    if (search_warps_per_cta(params->buckets, *cap) < 1)
        return bad("buckets/partition capacity exceed the search kernel's shared memory");
    return PHOBIC_OK;
}

uint64_t build_arena_bytes(const phobic_keys *keys, const phobic_params *params, const phobic_result *result,
                           bool debug) {
    uint64_t n = keys->n;
    uint64_t m = (n + params->partition_size - 1) / params->partition_size;
    uint64_t B = params->buckets;
    uint64_t t = 0;
    if (!keys->on_device) {
        if (keys->kind == PHOBIC_KEYS_STRINGS) t += align256(n ? keys->offsets[n] : 0) + align256(8 * (n + 1));
        else t += align256(key_bytes(keys));
    }
    t += align256(4 * kFulcrums);
    t += align256(4 * m) + align256(8 * ((m + kScanTile - 1) / kScanTile) + 8) + align256(8);
    t += align256(4 * n);                                              // rank
    if (keys->kind == PHOBIC_KEYS_STRINGS) t += align256(16 * n);      // mapped records
    t += align256(8 * n) + align256(2 * n) + align256(8 * n);          // lowers, bkt, sorted
    if (!result || !result->on_device) t += align256(4 * B * m) + align256(4 * (m + 1));
    if (debug) t += align256(16 * n) + align256(4 * m * B);
    return t + 4096;
}

// ------------------------------------------------------------------ build

struct PendingBuild {
    uint64_t n = 0;
    uint32_t partitions = 0, buckets = 0;
    uint32_t *d_pilots = nullptr, *d_off = nullptr;
    uint32_t *h_pilots = nullptr, *h_off = nullptr;
    unsigned long long *d_err = nullptr;
    uint4 *d_dbg_keys = nullptr;
    uint32_t *d_dbg_sizes = nullptr;
    DebugOut dbg;
};

phobic_status enqueue_build(Worker &w, const phobic_keys *keys, const phobic_params *params,
                            const phobic_result *result, const DebugOut *dbg, std::string *err) {
    uint32_t cap = 0, k_max = 0;
    phobic_status st = check_build_args(keys, params, &cap, &k_max, err);
    if (st != PHOBIC_OK) return st;
    if (!result || !result->pilots || !result->partition_offsets) {
        if (err) *err = "null result arrays";
        return PHOBIC_ERR_INVALID;
    }
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    const uint64_t n = keys->n;
    const uint32_t P = params->partition_size, B = params->buckets;
    const uint32_t m = (uint32_t)((n + P - 1) / P);  // mphf_builder.h:90
    const bool debug = dbg && (dbg->keys4 || dbg->bucket_sizes);

    PendingBuild pb;
    pb.n = n;
    pb.partitions = m;
    pb.buckets = B;
    if (debug) pb.dbg = *dbg;

    w.arena.reset();
    PHB_TRY(w.arena.reserve(build_arena_bytes(keys, params, result, debug)), "device arena");
    auto take = [&](size_t b) { return w.arena.take(b); };

    cudaStream_t s = w.stream;
    PHB_TRY(cudaEventRecord(w.ev[0], s), "event");

    // Inputs.
    KeyInput in{keys->data, keys->offsets};
    if (!keys->on_device && n) {
        if (keys->kind == PHOBIC_KEYS_STRINGS) {
            uint64_t nbytes = keys->offsets[n];
            void *d = take(nbytes);
            void *o = take(8 * (n + 1));
            if (nbytes) PHB_TRY(cudaMemcpyAsync(d, keys->data, nbytes, cudaMemcpyHostToDevice, s), "H2D keys");
            PHB_TRY(cudaMemcpyAsync(o, keys->offsets, 8 * (n + 1), cudaMemcpyHostToDevice, s), "H2D offsets");
            in = KeyInput{d, static_cast<const uint64_t *>(o)};
        } else {
            void *d = take(key_bytes(keys));
            PHB_TRY(cudaMemcpyAsync(d, keys->data, key_bytes(keys), cudaMemcpyHostToDevice, s), "H2D keys");
            in = KeyInput{d, nullptr};
        }
    }
    uint32_t *d_fulcs = static_cast<uint32_t *>(take(4 * kFulcrums));
    PHB_TRY(cudaMemcpyAsync(d_fulcs, params->fulcrums, 4 * kFulcrums, cudaMemcpyHostToDevice, s), "H2D fulcrums");

    uint32_t *d_count = static_cast<uint32_t *>(take(4 * (size_t)m));
    uint32_t tiles = (m + kScanTile - 1) / kScanTile;
    unsigned long long *d_tiles = static_cast<unsigned long long *>(take(8 * (size_t)tiles + 8));
    uint32_t *d_tile_ctr = reinterpret_cast<uint32_t *>(d_tiles + tiles);
    pb.d_err = static_cast<unsigned long long *>(take(8));
    uint32_t *d_rank = static_cast<uint32_t *>(take(4 * n));
    uint4 *d_mapped = keys->kind == PHOBIC_KEYS_STRINGS ? static_cast<uint4 *>(take(16 * n)) : nullptr;
    uint2 *d_lowers = static_cast<uint2 *>(take(8 * n));
    uint16_t *d_bkt = static_cast<uint16_t *>(take(2 * n));
    uint2 *d_sorted = static_cast<uint2 *>(take(8 * n));
    if (result->on_device) {
        pb.d_pilots = result->pilots;
        pb.d_off = result->partition_offsets;
    } else {
        pb.d_pilots = static_cast<uint32_t *>(take(4 * (size_t)B * m));
        pb.d_off = static_cast<uint32_t *>(take(4 * ((size_t)m + 1)));
        pb.h_pilots = result->pilots;
        pb.h_off = result->partition_offsets;
    }
    if (debug) {
        pb.d_dbg_keys = static_cast<uint4 *>(take(16 * n));
        pb.d_dbg_sizes = static_cast<uint32_t *>(take(4 * (size_t)m * B));
    }
    if (!d_sorted || !pb.d_off || (debug && !pb.d_dbg_sizes)) {
        if (err) *err = "arena sizing error";
        return PHOBIC_ERR_OOM;
    }

    PHB_TRY(cudaMemsetAsync(d_count, 0, 4 * (size_t)m, s), "memset");
    PHB_TRY(cudaMemsetAsync(d_tiles, 0, 8 * (size_t)tiles + 8, s), "memset");
    PHB_TRY(cudaMemsetAsync(pb.d_err, 0xFF, 8, s), "memset");
    if (m == 0) PHB_TRY(cudaMemsetAsync(pb.d_off, 0, 4, s), "memset");
    PHB_TRY(cudaEventRecord(w.ev[1], s), "event");

    const int grid_cap = w.sm_count * 8;
    const int grid = (int)std::min<uint64_t>((n + kMapThreads - 1) / kMapThreads, (uint64_t)grid_cap);
    if (n) {
        MapArgs ma{m, B, d_fulcs, d_count, d_rank, d_mapped, debug ? pb.d_dbg_keys : nullptr, pb.d_err};
        PHB_TRY(launch_map_count(keys->kind, in, n, ma, grid, s), "K1 map_count");
    }
    PHB_TRY(cudaEventRecord(w.ev[2], s), "event");
    ScanArgs sa{d_count, pb.d_off, m, cap, d_tiles, d_tile_ctr, pb.d_err};
    PHB_TRY(launch_scan(sa, s), "K2 scan");
    PHB_TRY(cudaEventRecord(w.ev[3], s), "event");
    if (n) {
        ScatterArgs xa{m, d_fulcs, pb.d_off, d_rank, d_mapped, d_lowers, d_bkt};
        PHB_TRY(launch_scatter(keys->kind, in, n, xa, grid, s), "K3 scatter");
    }
    PHB_TRY(cudaEventRecord(w.ev[4], s), "event");
    SearchArgs qa{pb.d_off, d_lowers, d_bkt, d_sorted, pb.d_pilots, debug ? pb.d_dbg_sizes : nullptr,
                  m, B, cap, k_max, pb.d_err};
    PHB_TRY(launch_search(qa, s), "K4 search");
    PHB_TRY(cudaEventRecord(w.ev[5], s), "event");

    PHB_TRY(cudaMemcpyAsync(w.pinned_err, pb.d_err, 8, cudaMemcpyDeviceToHost, s), "D2H status");
    if (!result->on_device) {
        if (m) PHB_TRY(cudaMemcpyAsync(pb.h_pilots, pb.d_pilots, 4 * (size_t)B * m, cudaMemcpyDeviceToHost, s), "D2H pilots");
        PHB_TRY(cudaMemcpyAsync(pb.h_off, pb.d_off, 4 * ((size_t)m + 1), cudaMemcpyDeviceToHost, s), "D2H offsets");
    }
    if (debug) {
        if (dbg->keys4 && n) PHB_TRY(cudaMemcpyAsync(dbg->keys4, pb.d_dbg_keys, 16 * n, cudaMemcpyDeviceToHost, s), "D2H keys");
        if (dbg->bucket_sizes && m)
            PHB_TRY(cudaMemcpyAsync(dbg->bucket_sizes, pb.d_dbg_sizes, 4 * (size_t)m * B, cudaMemcpyDeviceToHost, s), "D2H sizes");
    }
    PHB_TRY(cudaEventRecord(w.ev[6], s), "event");
    return PHOBIC_OK;
}

static float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    return ms;
}

phobic_status finish_build(Worker &w, phobic_timings *t, std::string *err) {
    phobic_status st = wait_event(w.ev[6], w.timeout_ms, err);
    if (st != PHOBIC_OK) return st;
    if (t) {
        t->input_transfer = elapsed(w.ev[0], w.ev[1]);
        t->bucket_sizes = elapsed(w.ev[1], w.ev[2]);
        t->partition_offsets = elapsed(w.ev[2], w.ev[3]);
        t->key_redistribution = elapsed(w.ev[3], w.ev[4]);
        t->search = elapsed(w.ev[4], w.ev[5]);
        t->result_transfer = elapsed(w.ev[5], w.ev[6]);
        t->total = elapsed(w.ev[0], w.ev[6]);
        t->kernels = 4;
    }
    unsigned long long e = *w.pinned_err;
    if (e == kNoError) return PHOBIC_OK;
    uint32_t code = (uint32_t)e, part = (uint32_t)(e >> 32);
    static const char *what[] = {"ok", "a bucket id is >= buckets (fulcrum table)", "oom",
                                 "a bucket holds more than 256 keys", "a partition exceeds max_partition_size",
                                 "pilot counter reached its limit", "bounded device wait expired", "cuda",
                                 "two keys of one bucket hash identically (duplicate keys)"};
    if (err) *err = std::string(code < 9 ? what[code] : "error") + " (partition " + std::to_string(part) + ")";
    return (phobic_status)code;
}

// ------------------------------------------------------------------ query

phobic_status run_query(Worker &w, const phobic_keys *keys, const phobic_params *params, uint32_t partitions,
                        const phobic_result *built, uint32_t *positions, uint64_t *bad, std::string *err) {
    if (!keys || !params || !built || (!positions && !bad)) {
        if (err) *err = "null argument";
        return PHOBIC_ERR_INVALID;
    }
    const uint64_t n = keys->n;
    const uint32_t B = params->buckets;
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    uint64_t bytes = 8192 + align256(4 * kFulcrums) + align256(8) + align256(4 * (size_t)B * partitions) +
                     align256(4 * ((size_t)partitions + 1)) + align256(4 * n) + align256(4 * ((n + 31) / 32 + 1));
    if (!keys->on_device)
        bytes += keys->kind == PHOBIC_KEYS_STRINGS ? align256(n ? keys->offsets[n] : 0) + align256(8 * (n + 1))
                                                   : align256(key_bytes(keys));
    w.arena.reset();
    PHB_TRY(w.arena.reserve(bytes), "device arena");
    cudaStream_t s = w.stream;
    KeyInput in{keys->data, keys->offsets};
    if (!keys->on_device && n) {
        if (keys->kind == PHOBIC_KEYS_STRINGS) {
            uint64_t nb = keys->offsets[n];
            void *d = w.arena.take(nb);
            void *o = w.arena.take(8 * (n + 1));
            if (nb) PHB_TRY(cudaMemcpyAsync(d, keys->data, nb, cudaMemcpyHostToDevice, s), "H2D keys");
            PHB_TRY(cudaMemcpyAsync(o, keys->offsets, 8 * (n + 1), cudaMemcpyHostToDevice, s), "H2D offsets");
            in = KeyInput{d, static_cast<const uint64_t *>(o)};
        } else {
            void *d = w.arena.take(key_bytes(keys));
            PHB_TRY(cudaMemcpyAsync(d, keys->data, key_bytes(keys), cudaMemcpyHostToDevice, s), "H2D keys");
            in = KeyInput{d, nullptr};
        }
    }
    uint32_t *d_fulcs = static_cast<uint32_t *>(w.arena.take(4 * kFulcrums));
    PHB_TRY(cudaMemcpyAsync(d_fulcs, params->fulcrums, 4 * kFulcrums, cudaMemcpyHostToDevice, s), "H2D fulcrums");
    unsigned long long *d_bad = static_cast<unsigned long long *>(w.arena.take(8));
    PHB_TRY(cudaMemsetAsync(d_bad, 0, 8, s), "memset");
    const uint32_t *d_pil = built->pilots, *d_off = built->partition_offsets;
    if (!built->on_device) {
        uint32_t *a = static_cast<uint32_t *>(w.arena.take(4 * (size_t)B * partitions));
        uint32_t *b = static_cast<uint32_t *>(w.arena.take(4 * ((size_t)partitions + 1)));
        PHB_TRY(cudaMemcpyAsync(a, built->pilots, 4 * (size_t)B * partitions, cudaMemcpyHostToDevice, s), "H2D pilots");
        PHB_TRY(cudaMemcpyAsync(b, built->partition_offsets, 4 * ((size_t)partitions + 1), cudaMemcpyHostToDevice, s),
                "H2D offsets");
        d_pil = a, d_off = b;
    }
    uint32_t n_built = 0;
    PHB_TRY(cudaMemcpyAsync(w.pinned_err, d_off + partitions, 4, cudaMemcpyDeviceToHost, s), "D2H n");
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    phobic_status st0 = wait_event(w.ev[7], w.timeout_ms, err);
    if (st0 != PHOBIC_OK) return st0;
    n_built = (uint32_t)*w.pinned_err;
    uint32_t *d_pos = nullptr;
    if (positions) d_pos = keys->on_device ? positions : static_cast<uint32_t *>(w.arena.take(4 * n));
    uint32_t *d_seen = nullptr;
    if (bad) {
        d_seen = static_cast<uint32_t *>(w.arena.take(4 * ((size_t)n_built / 32 + 1)));
        PHB_TRY(cudaMemsetAsync(d_seen, 0, 4 * ((size_t)n_built / 32 + 1), s), "memset");
    }
    QueryArgs qa{partitions, B, d_fulcs, d_pil, d_off, d_pos, d_seen, d_bad, n_built};
    int grid = (int)std::min<uint64_t>((n + kMapThreads - 1) / kMapThreads, (uint64_t)w.sm_count * 8);
    if (n && partitions) PHB_TRY(launch_query(keys->kind, in, n, qa, grid, s), "query");
    unsigned long long hbad = 0;
    if (bad) PHB_TRY(cudaMemcpyAsync(w.pinned_err, d_bad, 8, cudaMemcpyDeviceToHost, s), "D2H");
    if (positions && !keys->on_device && n)
        PHB_TRY(cudaMemcpyAsync(positions, d_pos, 4 * n, cudaMemcpyDeviceToHost, s), "D2H positions");
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    phobic_status st = wait_event(w.ev[7], w.timeout_ms, err);
    if (st != PHOBIC_OK) return st;
    if (bad) {
        hbad = *w.pinned_err;
        *bad = hbad + (n != n_built ? (n > n_built ? n - n_built : n_built - n) : 0);
    }
    return PHOBIC_OK;
}

}  // namespace phobicb200
