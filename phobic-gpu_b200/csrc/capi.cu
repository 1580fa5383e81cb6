// C ABI entry points (include/phobic_b200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"
#include "kernels.cuh"

using namespace phobicb200;

struct phobic_ctx {
    Worker w;
    std::string last_error;
    DeviceArena results;  // phobic_ctx_result
    DeviceArena encoded;  // phobic_encode_gpu output staging
};

extern "C" {

const char *phobic_status_string(phobic_status s) {
    switch (s) {
    case PHOBIC_OK: return "ok";
    case PHOBIC_ERR_INVALID: return "invalid argument";
    case PHOBIC_ERR_OOM: return "out of memory";
    case PHOBIC_ERR_BUCKET_OVERFLOW: return "bucket overflow (more than 256 keys)";
    case PHOBIC_ERR_PARTITION_OVERFLOW: return "partition overflow";
    case PHOBIC_ERR_SEARCH_LIMIT: return "pilot search limit reached";
    case PHOBIC_ERR_TIMEOUT: return "timeout";
    case PHOBIC_ERR_CUDA: return "cuda error";
    case PHOBIC_ERR_DUPLICATE_KEY: return "duplicate keys";
    case PHOBIC_ERR_BUDGET: return "request exceeds the memory budget";
    case PHOBIC_ERR_BUSY: return "queue full";
    case PHOBIC_ERR_NO_DEVICE: return "no suitable CUDA device";
    case PHOBIC_ERR_NOT_FOUND: return "unknown ticket";
    case PHOBIC_ERR_KEYS_CHANGED: return "keys changed during the build";
    }
    return "unknown status";
}

uint32_t phobic_partitions(uint64_t n, uint32_t partition_size) {
    if (!partition_size) return 0;
    return (uint32_t)((n + partition_size - 1) / partition_size);
}

// MPHFconfig (mphf_config.h:26-55) with the bucketers of bucketers.h:20-50.
// This translation unit is compiled with -ffp-contract=off: every double
// operation rounds on its own, so the table does not depend on FMA contraction.
phobic_status phobic_config(double lambda, uint32_t partition_size, int bucketer, int bucketer_ctor,
                            phobic_params *out) {
    if (!out || !(lambda > 0.0) || partition_size == 0 || bucketer < 0 || bucketer > 2) return PHOBIC_ERR_INVALID;
    double q = (double)partition_size / lambda;
    double bq = bucketer_ctor ? std::round(q) : std::ceil(q);
    if (!(bq >= 1.0) || bq > 65535.0) return PHOBIC_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    out->partition_size = partition_size;
    out->buckets = (uint32_t)bq;
    out->max_partition_size = default_max_partition(partition_size);
    const double c = 0.2 * lambda / std::sqrt((double)partition_size);  // OptBucketer::init
    const uint32_t top = out->buckets << 16;
    out->fulcrums[0] = 0;
    for (uint32_t xi = 1; xi < PHOBIC_FULCRUMS - 1; xi++) {
        double x = (double)xi / (double)(PHOBIC_FULCRUMS - 1);
        double y;
        if (bucketer == 1) y = x;
        else if (bucketer == 2) y = x < 0.6 ? x / 0.6 * 0.3 : 0.3 + (x - 0.6) / 0.4 * 0.7;
        else y = (x + (1.0 - x) * std::log(1.0 - x)) * (1.0 - c) + c * x;
        out->fulcrums[xi] = (uint32_t)(y * (double)top);
    }
    out->fulcrums[PHOBIC_FULCRUMS - 1] = top;
    return PHOBIC_OK;
}

phobic_status phobic_ctx_create(int device, phobic_ctx **out) {
    if (!out) return PHOBIC_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return PHOBIC_ERR_NO_DEVICE;
    }
    phobic_ctx *c = new phobic_ctx();
    std::string err;
    phobic_status st = c->w.init(device, &err);
    if (st != PHOBIC_OK) {
        c->w.destroy();
        delete c;
        return st;
    }
    *out = c;
    return PHOBIC_OK;
}

phobic_status phobic_ctx_destroy(phobic_ctx *ctx) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->w.destroy();
    delete ctx;
    return PHOBIC_OK;
}

const char *phobic_last_error(const phobic_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

uint64_t phobic_ctx_device_bytes(const phobic_ctx *ctx) { return ctx ? ctx->w.arena.capacity() : 0; }

phobic_status phobic_ctx_set_memory_limit(phobic_ctx *ctx, uint64_t bytes) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    if (cudaSetDevice(ctx->w.device) != cudaSuccess) {
        cudaGetLastError();
        return PHOBIC_ERR_CUDA;
    }
    ctx->w.arena.set_limit(bytes);
    return PHOBIC_OK;
}

void *phobic_ctx_stream(const phobic_ctx *ctx) { return ctx ? static_cast<void *>(ctx->w.stream) : nullptr; }

uint64_t phobic_build_bytes_needed(const phobic_keys *keys, const phobic_params *params) {
    if (!keys || !params || !params->partition_size) return 0;
    return sets_arena_bytes(keys, 1, params, nullptr, false);
}

phobic_status phobic_build(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                           const phobic_result *result, phobic_timings *timings) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    if (!keys || !result) {
        ctx->last_error = "null keys or result";
        return PHOBIC_ERR_INVALID;
    }
    phobic_status st = enqueue_sets(ctx->w, keys, 1, params, result, nullptr, &ctx->last_error);
    if (st != PHOBIC_OK) return st;
    return finish_sets(ctx->w, nullptr, timings, &ctx->last_error);
}

// Sets are built in groups of one key kind and placement whose keys sum to
// less than 2^32; each group is one launch of each kernel.
phobic_status phobic_build_batch(phobic_ctx *ctx, const phobic_keys *sets, uint32_t nsets,
                                 const phobic_params *params, const phobic_result *results,
                                 phobic_status *statuses, phobic_timings *timings) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    if (!sets || !results || !nsets) {
        ctx->last_error = "no key sets";
        return PHOBIC_ERR_INVALID;
    }
    std::vector<uint32_t> idx(nsets);
    for (uint32_t i = 0; i < nsets; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        return sets[a].kind * 2 + sets[a].on_device < sets[b].kind * 2 + sets[b].on_device;
    });
    if (timings) std::memset(timings, 0, sizeof(*timings));
    phobic_status first = PHOBIC_OK;
    std::vector<phobic_keys> gk;
    std::vector<phobic_result> gr;
    std::vector<uint32_t> gi;
    std::vector<phobic_status> gs;
    auto flush = [&]() -> phobic_status {
        if (gk.empty()) return PHOBIC_OK;
        gs.assign(gk.size(), PHOBIC_OK);
        phobic_timings t{};
        std::string err;
        phobic_status st = enqueue_sets(ctx->w, gk.data(), (uint32_t)gk.size(), params, gr.data(), nullptr, &err);
        if (st == PHOBIC_OK) st = finish_sets(ctx->w, gs.data(), &t, &err);
        else gs.assign(gk.size(), st);
        if (st != PHOBIC_OK && first == PHOBIC_OK) {
            first = st;
            ctx->last_error = err;
        }
        for (size_t j = 0; j < gk.size(); j++)
            if (statuses) statuses[gi[j]] = gs[j];
        if (timings) {
            timings->input_transfer += t.input_transfer;
            timings->bucket_sizes += t.bucket_sizes;
            timings->partition_offsets += t.partition_offsets;
            timings->key_redistribution += t.key_redistribution;
            timings->search += t.search;
            timings->result_transfer += t.result_transfer;
            timings->total += t.total;
            timings->kernels += t.kernels;
            timings->graph_replays += t.graph_replays;
        }
        gk.clear(), gr.clear(), gi.clear();
        return st;
    };
    uint64_t keys_in_group = 0;
    for (uint32_t j = 0; j < nsets; j++) {
        const phobic_keys &k = sets[idx[j]];
        bool same = !gk.empty() && gk[0].kind == k.kind && gk[0].on_device == k.on_device;
        if (!gk.empty() && (!same || keys_in_group + k.n > 0xFFFFFFFFull)) {
            flush();
            keys_in_group = 0;
        }
        gk.push_back(k);
        gr.push_back(results[idx[j]]);
        gi.push_back(idx[j]);
        keys_in_group += k.n;
    }
    flush();
    return first;
}

phobic_status phobic_build_u64(phobic_ctx *ctx, const uint64_t *keys, uint64_t n, const phobic_params *params,
                               uint32_t *pilots, uint32_t *partition_offsets, phobic_timings *timings) {
    phobic_keys k{PHOBIC_KEYS_U64, 0, n, keys, nullptr};
    phobic_result r{0, pilots, partition_offsets};
    return phobic_build(ctx, &k, params, &r, timings);
}

phobic_status phobic_build_strings(phobic_ctx *ctx, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                                   const phobic_params *params, uint32_t *pilots, uint32_t *partition_offsets,
                                   phobic_timings *timings) {
    phobic_keys k{PHOBIC_KEYS_STRINGS, 0, n, bytes, offsets};
    phobic_result r{0, pilots, partition_offsets};
    return phobic_build(ctx, &k, params, &r, timings);
}

phobic_status phobic_debug_build(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                                 const phobic_result *result, uint32_t *keys4, uint32_t *bucket_sizes) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    if (!keys || !result) return PHOBIC_ERR_INVALID;
    DebugOut dbg{keys4, bucket_sizes};
    phobic_status st = enqueue_sets(ctx->w, keys, 1, params, result, &dbg, &ctx->last_error);
    if (st != PHOBIC_OK) return st;
    return finish_sets(ctx->w, nullptr, nullptr, &ctx->last_error);
}

phobic_status phobic_debug_stalled_wait(phobic_ctx *ctx, uint32_t wait_ms, phobic_status *observed) {
    if (!ctx || !observed) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return run_stalled_wait(ctx->w, wait_ms, observed, &ctx->last_error);
}

phobic_status phobic_query(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params, uint32_t partitions,
                           const phobic_result *built, uint32_t *positions) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return run_query(ctx->w, keys, params, partitions, built, positions, nullptr, &ctx->last_error);
}

phobic_status phobic_encode_gpu(phobic_ctx *ctx, int pilot_encoder, int offset_encoder, const phobic_result *built,
                                uint32_t partitions, const phobic_params *params, uint8_t *out, size_t cap,
                                int out_on_device, size_t *size, double *bits_per_key) {
    if (!ctx) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return run_encode_gpu(ctx->w, ctx->encoded, pilot_encoder, offset_encoder, built, partitions, params, out, cap,
                          out_on_device, size, bits_per_key, &ctx->last_error);
}

phobic_status phobic_ctx_result(phobic_ctx *ctx, uint32_t buckets, uint32_t partitions, phobic_result *out) {
    if (!ctx || !out || buckets == 0) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    const size_t pb = align256(4 * (size_t)buckets * partitions), ob = align256(4 * ((size_t)partitions + 1));
    cudaError_t e = cudaSetDevice(ctx->w.device);
    if (e == cudaSuccess) e = ctx->results.reserve(pb + ob);
    if (e != cudaSuccess) return cuda_status(e, "phobic_ctx_result", &ctx->last_error);
    ctx->results.reset();
    out->on_device = 1;
    out->pilots = static_cast<uint32_t *>(ctx->results.take(pb));
    out->partition_offsets = static_cast<uint32_t *>(ctx->results.take(ob));
    return PHOBIC_OK;
}

phobic_status phobic_debug_checks(phobic_ctx *ctx, int *compiled, uint32_t *lines, int reset) {
    if (!ctx || !compiled || !lines) return PHOBIC_ERR_INVALID;
    if (cudaSetDevice(ctx->w.device) != cudaSuccess || cudaStreamSynchronize(ctx->w.stream) != cudaSuccess) {
        cudaGetLastError();
        return PHOBIC_ERR_CUDA;
    }
#ifdef PHOBIC_CHECKED
    *compiled = 1;
#else
    *compiled = 0;
#endif
    lines[0] = check_line_map(reset != 0);
    lines[1] = check_line_part(reset != 0);
    lines[2] = check_line_search(reset != 0);
    return PHOBIC_OK;
}

phobic_status phobic_ctx_set_tuning(phobic_ctx *ctx, const phobic_tuning *t) {
    if (!ctx || !t) return PHOBIC_ERR_INVALID;
    if (t->search_group != 0 && t->search_group != 1 && t->search_group != 2 && t->search_group != 4 &&
        t->search_group != 8)
        return PHOBIC_ERR_INVALID;
    if (t->search_pipeline > 1 || t->graphs_off > 1) return PHOBIC_ERR_INVALID;
    ctx->w.search_group = t->search_group;
    ctx->w.search_pipeline = t->search_pipeline;
    ctx->w.graphs_off = t->graphs_off;
    return PHOBIC_OK;
}

phobic_status phobic_autotune(phobic_ctx *ctx, const phobic_params *params, const char *path,
                              uint32_t *lines_written) {
    if (!ctx || !params) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return autotune(ctx->w, params, path, lines_written, &ctx->last_error);
}

phobic_status phobic_measure_int_peak(phobic_ctx *ctx, double *ops_per_s, double *kernel_ms) {
    if (!ctx || !ops_per_s || !kernel_ms) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return measure_int_peak(ctx->w, ops_per_s, kernel_ms, &ctx->last_error);
}

phobic_status phobic_ctx_kernel_arch(phobic_ctx *ctx, int *binary_version) {
    if (!ctx || !binary_version) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    return kernel_binary_version(ctx->w.device, binary_version, &ctx->last_error);
}

phobic_status phobic_verify(phobic_ctx *ctx, const phobic_keys *keys, const phobic_params *params,
                            const phobic_result *built, uint64_t *bad) {
    if (!ctx || !keys || !params || !bad) return PHOBIC_ERR_INVALID;
    ctx->last_error.clear();
    uint32_t partitions = phobic_partitions(keys->n, params->partition_size);
    return run_query(ctx->w, keys, params, partitions, built, nullptr, bad, &ctx->last_error);
}

}  // extern "C"
