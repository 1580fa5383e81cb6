// Build pipeline on one stream: the CUDA replacement of BuildInvocation::run
// (include/phobicGpu/mphf_builder.h:225-292).
//
//   reference stage (mphf_builder.h)           here
//   initialHash (host, :201-216)          ->  K1 map_count (XXH3 on the device)
//   input_transfer (:233-238)             ->  H2D of the raw keys (no 16-byte Key array)
//   bucket_sizes (:153-159)               ->  K1 (partition counts) + K4 (bucket counts)
//   bucket_sorting (:162-167)             ->  K4 (shared memory, per partition)
//   partition_offsets (:169-174)          ->  K2 decoupled-lookback scan
//   apply_partition_offsets (:176-180)    ->  K2 cursors + K3
//   key_redistribution (:182-187)         ->  K3 + K4
//   search (:189-194)                     ->  K4
//   result_transfer (:196-261)            ->  D2H of pilots and offsets
//
// A build takes a list of key sets; the plain build is the list of one.
#include "engine.hpp"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>

#include <omp.h>

#include "kernels.cuh"
#include "nvtx3/nvToolsExt.h"

namespace phobicb200 {

namespace {
// NVTX range for the host side of one stage (launches and copies), named with the
// reference's stage labels; profilers show it beside the kernels it launched.
struct StageRange {
    explicit StageRange(const char *name) { nvtxRangePushA(name); }
    ~StageRange() { nvtxRangePop(); }
};
}  // namespace

// ------------------------------------------------------------------ memory

cudaError_t DeviceArena::reserve(size_t bytes) {
    if (bytes <= cap_) return cudaSuccess;
    size_t want = align256(bytes);
    if (limit_ && want > limit_) return cudaErrorMemoryAllocation;
    release();
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

cudaError_t PinnedBuffer::reserve(size_t bytes) {
    if (bytes <= cap_) return cudaSuccess;
    release();
    cudaError_t e = cudaMallocHost(&p_, bytes);
    if (e != cudaSuccess) {
        p_ = nullptr;
        cudaGetLastError();
        return e;
    }
    cap_ = bytes;
    return cudaSuccess;
}

void PinnedBuffer::release() {
    if (p_) cudaFreeHost(p_);
    p_ = nullptr;
    cap_ = 0;
}

// ------------------------------------------------------------------ helpers

// True for host memory that is neither pinned nor registered with CUDA.
static bool is_pageable(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// Stage -> destination copies of finish_sets.  A large copy is split over a few host
// threads: writing fresh pageable memory is bound by page faults on one core.
static void copy_out(const std::vector<Worker::HostCopy> &copies, const char *stage) {
    constexpr size_t kSplitBytes = 4u << 20;
    constexpr int kParts = 4;
    for (const auto &c : copies) {
        char *dst = static_cast<char *>(c.dst);
        const char *src = stage + c.off;
        if (c.bytes < kSplitBytes) {
            std::memcpy(dst, src, c.bytes);
            continue;
        }
        const size_t part = (c.bytes / kParts + 4095) & ~size_t(4095);  // <= c.bytes
        std::vector<std::thread> helpers;
        size_t lo = part;  // first byte not handed to a helper
        for (int i = 1; i < kParts && lo < c.bytes; i++) {
            const size_t hi = std::min(c.bytes, lo + part);
            try {
                helpers.emplace_back([=] { std::memcpy(dst + lo, src + lo, hi - lo); });
            } catch (...) {  // no thread: this one copies the rest
                break;
            }
            lo = hi;
        }
        std::memcpy(dst, src, part);
        if (lo < c.bytes) std::memcpy(dst + lo, src + lo, c.bytes - lo);
        for (auto &h : helpers) h.join();
    }
}

// Host-to-device copy of `bytes` from host memory `src` on stream s.  Pinned (or small)
// sources are copied directly.  Pageable ones go in kUpChunk pieces through two pinned
// buffers: host threads fill one buffer while the copy engine drains the other, so the
// upload runs at host-memcpy speed (the driver's own pageable path reached 11 GB/s for
// 800 MB of keys, the pinned copy 55 GB/s).  Returns after the last piece is queued; the
// buffers are reused once their event has passed.
static constexpr size_t kUpChunk = 32u << 20;
static constexpr size_t kUpDirect = 4u << 20;

static phobic_status upload(Worker &w, void *dst, const void *src, size_t bytes, cudaStream_t s, std::string *err) {
    if (bytes < kUpDirect || !is_pageable(src) || w.up_stage.reserve(2 * kUpChunk) != cudaSuccess) {
        cudaGetLastError();
        PHB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D keys");
        return PHOBIC_OK;
    }
    const int threads = std::max(1, std::min(8, omp_get_max_threads()));
    char *stage = static_cast<char *>(w.up_stage.data());
    for (size_t off = 0, i = 0; off < bytes; off += kUpChunk, i++) {
        const size_t len = std::min(kUpChunk, bytes - off);
        const int b = (int)(i & 1);
        phobic_status st = wait_event(w.up_ev[b], w.timeout_ms, err);  // the buffer's previous copy is done
        if (st != PHOBIC_OK) return st;
        char *buf = stage + b * kUpChunk;
        const char *from = static_cast<const char *>(src) + off;
        const int64_t pieces = (int64_t)((len + (1u << 20) - 1) >> 20);
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int64_t q = 0; q < pieces; q++) {
            const size_t lo = (size_t)q << 20, hi = std::min(len, lo + (1u << 20));
            std::memcpy(buf + lo, from + lo, hi - lo);
        }
        PHB_TRY(cudaMemcpyAsync(static_cast<char *>(dst) + off, buf, len, cudaMemcpyHostToDevice, s), "H2D keys");
        PHB_TRY(cudaEventRecord(w.up_ev[b], s), "event");
    }
    return PHOBIC_OK;
}

// Device-to-host copy of `bytes` into host memory `dst`, complete when this returns (the
// stream's earlier work included).  Pageable destinations are served in kUpChunk pieces
// through the two pinned buffers: the copy engine fills one while host threads empty the
// other.
static phobic_status download(Worker &w, void *dst, const void *src, size_t bytes, cudaStream_t s, std::string *err) {
    const bool staged = bytes >= kUpDirect && is_pageable(dst) && w.up_stage.reserve(2 * kUpChunk) == cudaSuccess;
    cudaGetLastError();
    if (!staged) {
        PHB_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "D2H");
        PHB_TRY(cudaEventRecord(w.up_ev[0], s), "event");
        return wait_event(w.up_ev[0], w.timeout_ms, err);
    }
    const int threads = std::max(1, std::min(8, omp_get_max_threads()));
    char *stage = static_cast<char *>(w.up_stage.data());
    const size_t chunks = (bytes + kUpChunk - 1) / kUpChunk;
    auto issue = [&](size_t i) -> phobic_status {
        const size_t off = i * kUpChunk, len = std::min(kUpChunk, bytes - off);
        const int b = (int)(i & 1);
        phobic_status st = wait_event(w.up_ev[b], w.timeout_ms, err);  // an earlier upload's copy is done
        if (st != PHOBIC_OK) return st;
        PHB_TRY(cudaMemcpyAsync(stage + b * kUpChunk, static_cast<const char *>(src) + off, len,
                                cudaMemcpyDeviceToHost, s), "D2H");
        PHB_TRY(cudaEventRecord(w.up_ev[b], s), "event");
        return PHOBIC_OK;
    };
    phobic_status st = issue(0);
    if (st == PHOBIC_OK && chunks > 1) st = issue(1);
    for (size_t i = 0; st == PHOBIC_OK && i < chunks; i++) {
        const int b = (int)(i & 1);
        if ((st = wait_event(w.up_ev[b], w.timeout_ms, err)) != PHOBIC_OK) break;
        const size_t off = i * kUpChunk, len = std::min(kUpChunk, bytes - off);
        const char *buf = stage + b * kUpChunk;
        char *to = static_cast<char *>(dst) + off;
        const int64_t pieces = (int64_t)((len + (1u << 20) - 1) >> 20);
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int64_t q = 0; q < pieces; q++) {
            const size_t lo = (size_t)q << 20, hi = std::min(len, lo + (1u << 20));
            std::memcpy(to + lo, buf + lo, hi - lo);
        }
        if (i + 2 < chunks) st = issue(i + 2);
    }
    return st;
}

phobic_status cuda_status(cudaError_t e, const char *what, std::string *err) {
    if (e == cudaSuccess) return PHOBIC_OK;
    if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return PHOBIC_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return PHOBIC_ERR_NO_DEVICE;
    return PHOBIC_ERR_CUDA;
}


// Polls `done` (a cudaEventQuery / cudaStreamQuery) until it succeeds, fails or the
// bound passes: yields for the first 2000 polls, then sleeps 50 us between polls, so a
// long build does not hold a host core.
template <typename Query>
static phobic_status bounded_wait(Query done, uint64_t timeout_ms, std::string *err) {
    auto t0 = std::chrono::steady_clock::now();
    uint32_t polls = 0;
    for (;;) {
        cudaError_t e = done();
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

phobic_status wait_event(cudaEvent_t ev, uint64_t timeout_ms, std::string *err) {
    return bounded_wait([ev] { return cudaEventQuery(ev); }, timeout_ms, err);
}

phobic_status wait_stream(cudaStream_t s, uint64_t timeout_ms, std::string *err) {
    return bounded_wait([s] { return cudaStreamQuery(s); }, timeout_ms, err);
}

uint64_t env_timeout_ms() {
    if (const char *t = std::getenv("PHOBIC_TIMEOUT_MS")) {
        char *end = nullptr;
        const unsigned long long v = std::strtoull(t, &end, 10);
        if (end != t && v) return v;
    }
    return 120000;
}

namespace {
std::mutex g_key_change_mu;
bool g_key_change_armed = false;
uint64_t g_key_change_index = 0, g_key_change_mask = 0;
}  // namespace

void set_key_change(uint64_t index, uint64_t mask) {
    std::lock_guard<std::mutex> lk(g_key_change_mu);
    g_key_change_armed = mask != 0;
    g_key_change_index = index;
    g_key_change_mask = mask;
}

bool take_key_change(uint64_t n, int kind, uint64_t *index, uint64_t *mask) {
    std::lock_guard<std::mutex> lk(g_key_change_mu);
    if (!g_key_change_armed || kind != PHOBIC_KEYS_U64 || g_key_change_index >= n) return false;
    g_key_change_armed = false;
    *index = g_key_change_index;
    *mask = g_key_change_mask;
    return true;
}

uint32_t default_max_partition(uint32_t P) {
    uint32_t words = (P + P / 2) / 32;  // mphf_config.h:61-64, 32 slots per bitmap word (search.comp:21)
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
    for (auto &e : up_ev) PHB_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    PHB_TRY(pinned.reserve(1 << 16), "cudaMallocHost");
    timeout_ms = env_timeout_ms();
    return PHOBIC_OK;
}

void Worker::drop_graph() {
    // An executable graph still in flight is freed when its launch completes.
    if (graph_exec) cudaGraphExecDestroy(graph_exec), graph_exec = nullptr;
    graph_key.clear();
}

void Worker::destroy() {
    if (stream) {
        cudaSetDevice(device);
        if (ev[7] && cudaEventRecord(ev[7], stream) == cudaSuccess) wait_event(ev[7], timeout_ms, nullptr);
    }
    drop_graph();
    arena.release();
    pinned.release();
    stage.release();
    pending_copies.clear();
    up_stage.release();
    for (auto &e : ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (auto &e : up_ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    if (stream) cudaStreamDestroy(stream), stream = nullptr;
}

// ------------------------------------------------------------------ validation and sizes

static uint64_t key_bytes(const phobic_keys *k) {
    switch (k->kind) {
    case PHOBIC_KEYS_U64: return 8 * k->n;
    case PHOBIC_KEYS_BYTES16:
    case PHOBIC_KEYS_PREHASHED: return 16 * k->n;
    default: return 0;
    }
}

static uint64_t staged_bytes(const phobic_keys *k) {
    if (k->on_device) return 0;
    if (k->kind == PHOBIC_KEYS_STRINGS) return align256(k->n ? k->offsets[k->n] : 0) + align256(8 * (k->n + 1));
    return align256(key_bytes(k));
}

phobic_status check_keys(const phobic_keys *keys, std::string *err) {
    auto bad = [&](const char *m) {
        if (err) *err = m;
        return PHOBIC_ERR_INVALID;
    };
    if (!keys) return bad("null keys");
    if (keys->kind < PHOBIC_KEYS_U64 || keys->kind > PHOBIC_KEYS_STRINGS) return bad("unknown key kind");
    if (keys->n > 0xFFFFFFFFull) return bad("more than 2^32-1 keys (the reference's uint32 size, mphf_builder.h:56)");
    if (keys->kind == PHOBIC_KEYS_STRINGS && keys->n && !keys->offsets) return bad("strings need offsets");
    if (keys->kind != PHOBIC_KEYS_STRINGS && keys->n && !keys->data) return bad("null key data");
    if (keys->on_device && keys->n) {
        // The kernels read u64 keys and 16-byte records as 8-byte words, Keys as 4-byte
        // words, and string offsets as 8-byte words.
        uintptr_t d = reinterpret_cast<uintptr_t>(keys->data), o = reinterpret_cast<uintptr_t>(keys->offsets);
        if ((keys->kind == PHOBIC_KEYS_U64 || keys->kind == PHOBIC_KEYS_BYTES16) && (d & 7))
            return bad("device keys must be 8-byte aligned");
        if (keys->kind == PHOBIC_KEYS_PREHASHED && (d & 3)) return bad("device Key records must be 4-byte aligned");
        if (keys->kind == PHOBIC_KEYS_STRINGS && (o & 7)) return bad("device string offsets must be 8-byte aligned");
    }
    return PHOBIC_OK;
}

phobic_status check_params(const phobic_params *params, uint32_t *cap, uint32_t *k_max, std::string *err) {
    auto bad = [&](const char *m) {
        if (err) *err = m;
        return PHOBIC_ERR_INVALID;
    };
    if (!params) return bad("null params");
    if (params->partition_size == 0) return bad("partition_size must be > 0");
    if (params->buckets == 0 || params->buckets > 65535) return bad("buckets must be in 1..65535");
    if (params->fulcrums[kFulcrums - 1] != (params->buckets << 16))
        return bad("fulcrum table does not end at buckets << 16 (mphf_config.h:54)");
    *cap = params->max_partition_size ? params->max_partition_size : default_max_partition(params->partition_size);
    *k_max = params->max_pilot_counter ? params->max_pilot_counter : kDefaultMaxPilot;
    if (*cap > 65535) return bad("max_partition_size must be <= 65535");
    if (search_warps_per_cta(params->buckets, *cap) < 1)
        return bad("buckets/partition capacity exceed the search kernel's shared memory");
    return PHOBIC_OK;
}

uint64_t sets_arena_bytes(const phobic_keys *sets, uint32_t nsets, const phobic_params *params,
                          const phobic_result *results, bool debug) {
    const uint64_t P = params->partition_size, B = params->buckets;
    uint64_t N = 0, M = 0, t = 0;
    for (uint32_t s = 0; s < nsets; s++) {
        uint64_t m = (sets[s].n + P - 1) / P;
        N += sets[s].n;
        M += m;
        t += staged_bytes(&sets[s]);
        if (!results || !results[s].on_device) t += align256(4 * B * m) + align256(4 * (m + 1));
    }
    t += align256(4 * kFulcrums) + align256(sizeof(SetDesc) * nsets) + 2 * align256(8 * (nsets + 1)) +
         align256(8 * nsets) + align256(64);
    const uint64_t MS = M * plan_map(N, M, 0).stride;  // count matrix entries
    t += align256(4 * MS) + align256(4 * (MS + 1)) + align256(8 * ((MS + kScanTile - 1) / kScanTile) + 8);
    if (nsets && sets[0].kind == PHOBIC_KEYS_STRINGS) t += align256(16 * N);
    // lowers, bucket ids, partition records (also the search's scratch), cursors
    t += align256(8 * N) + align256(2 * N) + align256(16 * N) + align256(4 * M) + align256(4 * kMaxBins);
    if (debug) t += align256(16 * N) + align256(4 * M * B);
    return t + 4096;
}

// ------------------------------------------------------------------ build

// Largest build (in partitions) whose stages are replayed as a graph.  Measured on the B200
// with device-resident keys and results (per build, graph against stage-by-stage launches):
// 10^4 keys 0.387 against 0.396 ms, 10^6 keys (489 partitions) 0.4675 against 0.4745 ms, and
// 10^7 keys (4,000 partitions) 1.933 against 1.917 ms, so large builds launch stage by stage.
constexpr uint64_t kGraphMaxPartitions = 2048;

phobic_status enqueue_sets(Worker &w, const phobic_keys *sets, uint32_t nsets, const phobic_params *params,
                           const phobic_result *results, const DebugOut *dbg, std::string *err) {
    uint32_t cap = 0, k_max = 0;
    phobic_status st = check_params(params, &cap, &k_max, err);
    if (st != PHOBIC_OK) return st;
    if (!sets || !results || nsets == 0) {
        if (err) *err = "no key sets";
        return PHOBIC_ERR_INVALID;
    }
    const int kind = sets[0].kind;
    const int on_dev = sets[0].on_device;
    uint64_t N = 0, M = 0;
    const uint32_t P = params->partition_size, B = params->buckets;
    for (uint32_t s = 0; s < nsets; s++) {
        if ((st = check_keys(&sets[s], err)) != PHOBIC_OK) return st;
        if (sets[s].kind != kind || sets[s].on_device != on_dev) {
            if (err) *err = "all sets of one build must share key kind and placement";
            return PHOBIC_ERR_INVALID;
        }
        const phobic_result &r = results[s];
        if (!r.partition_offsets || (!r.pilots && sets[s].n)) {
            if (err) *err = "null result arrays";
            return PHOBIC_ERR_INVALID;
        }
        if (r.on_device && ((reinterpret_cast<uintptr_t>(r.pilots) | reinterpret_cast<uintptr_t>(r.partition_offsets)) & 3)) {
            if (err) *err = "device result arrays must be 4-byte aligned";
            return PHOBIC_ERR_INVALID;
        }
        N += sets[s].n;
        M += (sets[s].n + P - 1) / P;
    }
    const MapPlan plan = plan_map(N, M, w.sm_count);
    if (N > 0xFFFFFFFFull || M * plan.stride > 0xFFFFFFFFull) {
        if (err) *err = "a build holds at most 2^32-1 keys in total";
        return PHOBIC_ERR_INVALID;
    }
    const bool debug = dbg && (dbg->keys4 || dbg->bucket_sizes) && nsets == 1;
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");

    // Host-side set table (pinned): SetDesc[nsets] | key_base[nsets+1] | part_base[nsets+1] |
    // fulcrums | err[nsets].  Everything before err goes up in one copy to the same layout on
    // the device.
    const size_t tab_desc = align256(sizeof(SetDesc) * nsets), tab_kb = align256(8 * (nsets + 1)),
                 tab_pb = align256(8 * (nsets + 1)), tab_fulcs = align256(4 * kFulcrums), tab_err = align256(8 * nsets);
    const size_t tab_in = tab_desc + tab_kb + tab_pb + tab_fulcs;
    PHB_TRY(w.pinned.reserve(tab_in + tab_err), "pinned table");
    char *tab = static_cast<char *>(w.pinned.data());
    SetDesc *hdesc = reinterpret_cast<SetDesc *>(tab);
    uint64_t *hkb = reinterpret_cast<uint64_t *>(tab + tab_desc);
    uint32_t *hpb = reinterpret_cast<uint32_t *>(tab + tab_desc + tab_kb);
    std::memcpy(tab + tab_desc + tab_kb + tab_pb, params->fulcrums, 4 * kFulcrums);
    w.pending_err = reinterpret_cast<unsigned long long *>(tab + tab_in);
    w.pending_sets = nsets;

    // Host results: pinned destinations are copied to directly, pageable ones through the
    // worker's pinned stage (sized here, before any launch, since growing it reallocates).
    w.pending_copies.clear();
    size_t stage_bytes = 0;
    for (uint32_t i = 0; i < nsets; i++) {
        if (results[i].on_device) continue;
        const uint64_t parts = (sets[i].n + P - 1) / P;
        const std::pair<void *, size_t> arrays[2] = {{results[i].pilots, parts ? 4 * (size_t)B * parts : 0},
                                                      {results[i].partition_offsets, 4 * ((size_t)parts + 1)}};
        for (const auto &a : arrays)
            if (a.second && is_pageable(a.first)) {
                w.pending_copies.push_back(Worker::HostCopy{a.first, stage_bytes, a.second});
                stage_bytes += align256(a.second);
            }
    }
    if (stage_bytes && w.stage.reserve(stage_bytes) != cudaSuccess) {
        cudaGetLastError();
        w.pending_copies.clear();  // no pinned memory to be had: copy to pageable memory directly
    }

    w.arena.reset();
    PHB_TRY(w.arena.reserve(sets_arena_bytes(sets, nsets, params, results, debug)), "device arena");
    auto take = [&](size_t b) { return w.arena.take(b); };
    cudaStream_t s = w.stream;
    PHB_TRY(cudaEventRecord(w.ev[0], s), "event");

    // Inputs and per-set descriptors.
    uint64_t kb = 0;
    uint32_t pb = 0;
    for (uint32_t i = 0; i < nsets; i++) {
        const phobic_keys &k = sets[i];
        SetDesc &d = hdesc[i];
        std::memset(&d, 0, sizeof(d));
        d.data = k.data;
        d.offsets = k.offsets;
        if (!k.on_device && k.n) {
            if (kind == PHOBIC_KEYS_STRINGS) {
                uint64_t nb = k.offsets[k.n];
                void *dd = take(nb);
                void *oo = take(8 * (k.n + 1));
                phobic_status ust = nb ? upload(w, dd, k.data, nb, s, err) : PHOBIC_OK;
                if (ust == PHOBIC_OK) ust = upload(w, oo, k.offsets, 8 * (k.n + 1), s, err);
                if (ust != PHOBIC_OK) return ust;
                d.data = dd;
                d.offsets = static_cast<const uint64_t *>(oo);
            } else {
                void *dd = take(key_bytes(&k));
                const phobic_status ust = upload(w, dd, k.data, key_bytes(&k), s, err);
                if (ust != PHOBIC_OK) return ust;
                d.data = dd;
            }
        }
        const uint32_t m = (uint32_t)((k.n + P - 1) / P);  // mphf_builder.h:90
        d.key_base = kb;
        d.n = (uint32_t)k.n;
        d.part_base = pb;
        d.partitions = m;
        if (results[i].on_device) {
            d.pilots = results[i].pilots;
            d.part_off = results[i].partition_offsets;
        } else {
            d.pilots = static_cast<uint32_t *>(take(4 * (size_t)B * m));
            d.part_off = static_cast<uint32_t *>(take(4 * ((size_t)m + 1)));
        }
        if (m == 0) PHB_TRY(cudaMemsetAsync(d.part_off, 0, 4, s), "memset");
        hkb[i] = kb;
        hpb[i] = pb;
        kb += k.n;
        pb += m;
    }
    hkb[nsets] = kb;
    hpb[nsets] = pb;
    char *d_tab = static_cast<char *>(take(tab_in));
    SetDesc *d_desc = reinterpret_cast<SetDesc *>(d_tab);
    uint64_t *d_kb = reinterpret_cast<uint64_t *>(d_tab + tab_desc);
    uint32_t *d_pb = reinterpret_cast<uint32_t *>(d_tab + tab_desc + tab_kb);
    uint32_t *d_fulcs = reinterpret_cast<uint32_t *>(d_tab + tab_desc + tab_kb + tab_pb);
    unsigned long long *d_err = static_cast<unsigned long long *>(take(8 * nsets));
    uint32_t *d_queue = static_cast<uint32_t *>(take(64));
    const uint64_t MS = M * plan.stride;  // count matrix entries
    uint32_t *d_count = static_cast<uint32_t *>(take(4 * MS));
    uint32_t *d_G = static_cast<uint32_t *>(take(4 * (MS + 1)));
    const uint32_t tiles = (uint32_t)((MS + kScanTile - 1) / kScanTile);
    unsigned long long *d_tiles = static_cast<unsigned long long *>(take(8 * (size_t)tiles + 8));
    uint4 *d_mapped = kind == PHOBIC_KEYS_STRINGS ? static_cast<uint4 *>(take(16 * N)) : nullptr;
    uint2 *d_lowers = static_cast<uint2 *>(take(8 * N));
    uint16_t *d_bkt = static_cast<uint16_t *>(take(2 * N));
    uint4 *d_inter = static_cast<uint4 *>(take(16 * N));
    uint2 *d_sorted = reinterpret_cast<uint2 *>(d_inter);  // K4 scratch, after K3 is done with d_inter
    uint32_t *d_pcur = static_cast<uint32_t *>(take(4 * M));
    uint32_t *d_bincur = static_cast<uint32_t *>(take(4 * kMaxBins));
    uint4 *d_dbg_keys = debug ? static_cast<uint4 *>(take(16 * N)) : nullptr;
    uint32_t *d_dbg_sizes = debug ? static_cast<uint32_t *>(take(4 * M * B)) : nullptr;
    if (!d_bincur || (debug && !d_dbg_sizes)) {
        if (err) *err = "arena sizing error";
        return PHOBIC_ERR_OOM;
    }
    PHB_TRY(cudaMemcpyAsync(d_tab, tab, tab_in, cudaMemcpyHostToDevice, s), "H2D set table and fulcrums");
    uint64_t kc_index = 0, kc_mask = 0;
    const bool key_change = nsets == 1 && take_key_change(N, kind, &kc_index, &kc_mask);
    const uint32_t wshift = part_wshift(M);
    const SearchShape shape = choose_search_shape(w, params, (uint32_t)M);
    MapArgs ma{d_desc, d_kb, nsets, B, N, d_fulcs, d_count, d_mapped, d_dbg_keys, d_lowers, d_bkt, d_err,
               (uint32_t)M, plan.stride, plan.chunk};
    ScanArgs sa{d_count, d_G, nullptr, (uint32_t)MS, d_tiles, reinterpret_cast<uint32_t *>(d_tiles + tiles), nsets,
                d_err, 0};
    PartArgs pa{d_inter, d_bincur, d_pcur, wshift, (uint32_t)((M + (1ull << wshift) - 1) >> wshift), (uint32_t)M};
    SearchArgs qa{d_desc, d_pb, nsets, (uint32_t)M, d_G, plan.stride, d_lowers, d_bkt, d_sorted, d_dbg_sizes, B, cap,
                  k_max, d_queue, d_err, d_pcur};

    // The device stages, from the per-build memsets to the status copy: enqueued one by one,
    // or under stream capture (the stage events then become event-record nodes of the graph).
    auto stages = [&](bool capture) -> phobic_status {
        auto record = [&](cudaEvent_t e) {
            return capture ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
        };
        PHB_TRY(cudaMemsetAsync(d_err, 0xFF, 8 * nsets, s), "memset");
        PHB_TRY(cudaMemsetAsync(d_queue, 0, 64, s), "memset");
        PHB_TRY(cudaMemsetAsync(d_count, 0, 4 * MS, s), "memset");
        PHB_TRY(cudaMemsetAsync(d_tiles, 0, 8 * (size_t)tiles + 8, s), "memset");
        if (M == 0) PHB_TRY(cudaMemsetAsync(d_G, 0, 4, s), "memset");
        PHB_TRY(record(w.ev[1]), "event");
        // K1, scan, size check, two partition passes, search; none when there are no keys.
        {
            StageRange r("bucket_sizes (K1)");
            PHB_TRY(launch_map_count(kind, ma, plan, s), "K1 map_count");
        }
        if (key_change)
            PHB_TRY(launch_change_key(const_cast<void *>(hdesc[0].data), kc_index, kc_mask, s), "key change");
        PHB_TRY(record(w.ev[2]), "event");
        {
            StageRange r("partition_offsets (K2)");
            PHB_TRY(launch_scan(sa, s), "K2 scan");
        }
        PHB_TRY(launch_check_sizes(d_G, (uint32_t)M, plan.stride, cap, d_pb, nsets, d_err, &pa, s), "K2 size check");
        PHB_TRY(record(w.ev[3]), "event");
        {
            StageRange r("key_redistribution (K3)");
            PHB_TRY(launch_partition(kind, ma, pa, w.sm_count, s), "K3 partition");
        }
        PHB_TRY(record(w.ev[4]), "event");
        {
            StageRange r("search (K4)");
            PHB_TRY(launch_search(qa, w.sm_count, s, shape), "K4 search");
        }
        PHB_TRY(record(w.ev[5]), "event");
        PHB_TRY(cudaMemcpyAsync(w.pending_err, d_err, 8 * nsets, cudaMemcpyDeviceToHost, s), "D2H status");
        return PHOBIC_OK;
    };
    w.pending_kernels = N ? 6 : 0;
    w.pending_graph = false;
    cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;
    if (w.graphs_off || debug || key_change || !N || M > kGraphMaxPartitions ||
        cudaStreamIsCapturing(s, &cap_status) != cudaSuccess || cap_status != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        w.drop_graph();  // also when the caller is capturing the stream: the stages join that capture
    } else {
        // Everything the launches depend on: sizes, parameters, plan, shape and every buffer.
        std::vector<uint64_t> key{nsets, (uint64_t)kind, N, M, B, cap, k_max, plan.stride, plan.chunk, plan.grid,
                                  (uint64_t)plan.chunked | (uint64_t)plan.narrow << 1, wshift, tiles,
                                  (uint64_t)shape.group, (uint64_t)shape.pipeline, (uint64_t)w.sm_count};
        for (const void *p : {(const void *)d_fulcs, (const void *)d_desc, (const void *)d_kb, (const void *)d_pb,
                              (const void *)d_err, (const void *)d_queue, (const void *)d_count, (const void *)d_G,
                              (const void *)d_tiles, (const void *)d_mapped, (const void *)d_lowers,
                              (const void *)d_bkt, (const void *)d_inter, (const void *)d_pcur, (const void *)d_bincur,
                              (const void *)w.pending_err})
            key.push_back((uint64_t)reinterpret_cast<uintptr_t>(p));
        const size_t desc_words = (sizeof(SetDesc) * nsets + 7) / 8;
        key.resize(key.size() + desc_words, 0);
        std::memcpy(key.data() + key.size() - desc_words, hdesc, sizeof(SetDesc) * nsets);
        if (key != w.graph_key) {
            w.drop_graph();
            w.graph_key = std::move(key);
        } else if (!w.graph_exec) {  // the second build in a row with these launches: capture it
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const phobic_status cst = stages(true);
                cudaGraph_t g = nullptr;
                const cudaError_t ee = cudaStreamEndCapture(s, &g);
                if (cst == PHOBIC_OK && ee == cudaSuccess && g &&
                    cudaGraphInstantiate(&w.graph_exec, g, 0) != cudaSuccess)
                    w.graph_exec = nullptr;
                if (g) cudaGraphDestroy(g);
            }
            cudaGetLastError();  // a capture that failed leaves nothing enqueued: launch one by one
        }
        if (w.graph_exec) {
            if (cudaGraphLaunch(w.graph_exec, s) == cudaSuccess) {
                w.pending_graph = true;
            } else {  // launched stage by stage below, which reports a lasting error
                cudaGetLastError();
                w.drop_graph();
            }
        }
    }
    if (!w.pending_graph) {
        const phobic_status sst = stages(false);
        if (sst != PHOBIC_OK) return sst;
    }
    {
        size_t next = 0;  // pending_copies are in the order of the arrays below
        char *stage = static_cast<char *>(w.stage.data());
        auto to_host = [&](void *dst, const void *src, size_t bytes) {
            if (next < w.pending_copies.size() && w.pending_copies[next].dst == dst)
                dst = stage + w.pending_copies[next++].off;
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        };
        for (uint32_t i = 0; i < nsets; i++) {
            if (results[i].on_device) continue;
            const SetDesc &d = hdesc[i];
            if (d.partitions) PHB_TRY(to_host(results[i].pilots, d.pilots, 4 * (size_t)B * d.partitions), "D2H pilots");
            PHB_TRY(to_host(results[i].partition_offsets, d.part_off, 4 * ((size_t)d.partitions + 1)), "D2H offsets");
        }
    }
    if (debug) {
        if (dbg->keys4 && N) PHB_TRY(cudaMemcpyAsync(dbg->keys4, d_dbg_keys, 16 * N, cudaMemcpyDeviceToHost, s), "D2H keys");
        if (dbg->bucket_sizes && M)
            PHB_TRY(cudaMemcpyAsync(dbg->bucket_sizes, d_dbg_sizes, 4 * M * B, cudaMemcpyDeviceToHost, s), "D2H sizes");
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

static const char *error_text(uint32_t code) {
    switch (code) {
    case PHOBIC_ERR_INVALID: return "a bucket id is >= buckets (fulcrum table)";
    case PHOBIC_ERR_BUCKET_OVERFLOW: return "a bucket holds more than 256 keys";
    case PHOBIC_ERR_PARTITION_OVERFLOW: return "a partition exceeds max_partition_size";
    case PHOBIC_ERR_SEARCH_LIMIT: return "pilot counter reached its limit";
    case PHOBIC_ERR_TIMEOUT: return "bounded device wait expired";
    case PHOBIC_ERR_DUPLICATE_KEY: return "two keys of one bucket hash identically (duplicate keys)";
    case PHOBIC_ERR_KEYS_CHANGED:
        return "the passes of the build read different keys (device keys written while the build ran)";
    default: return "error";
    }
}

phobic_status finish_sets(Worker &w, phobic_status *statuses, phobic_timings *t, std::string *err) {
    phobic_status st;
    {
        StageRange r("wait for the build");
        st = wait_event(w.ev[6], w.timeout_ms, err);
    }
    if (st != PHOBIC_OK) return st;
    if (!w.pending_copies.empty()) {
        StageRange r("copy results to pageable memory");
        copy_out(w.pending_copies, static_cast<const char *>(w.stage.data()));
        w.pending_copies.clear();
    }
    if (t) {
        t->input_transfer = elapsed(w.ev[0], w.ev[1]);
        t->bucket_sizes = elapsed(w.ev[1], w.ev[2]);
        t->partition_offsets = elapsed(w.ev[2], w.ev[3]);
        t->key_redistribution = elapsed(w.ev[3], w.ev[4]);
        t->search = elapsed(w.ev[4], w.ev[5]);
        t->result_transfer = elapsed(w.ev[5], w.ev[6]);
        t->total = elapsed(w.ev[0], w.ev[6]);
        t->kernels = w.pending_kernels;
        t->graph_replays = w.pending_graph ? 1u : 0u;
    }
    phobic_status first = PHOBIC_OK;
    for (uint32_t i = 0; i < w.pending_sets; i++) {
        unsigned long long e = w.pending_err[i];
        phobic_status si = e == kNoError ? PHOBIC_OK : (phobic_status)(uint32_t)e;
        if (statuses) statuses[i] = si;
        if (si != PHOBIC_OK && first == PHOBIC_OK) {
            first = si;
            if (err)
                *err = std::string(error_text((uint32_t)e)) + " (set " + std::to_string(i) + ", partition " +
                       std::to_string((uint32_t)(e >> 32)) + ")";
        }
    }
    return first;
}

// ------------------------------------------------------------------ bounded-wait test

phobic_status run_stalled_wait(Worker &w, uint32_t wait_ms, phobic_status *observed, std::string *err) {
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    const uint32_t m = 2 * kScanTile;  // two tiles: tile 1 waits on tile 0, which never runs
    w.arena.reset();
    PHB_TRY(w.arena.reserve(align256(4 * m) + align256(4 * (m + 1)) + align256(8 * 2 + 8) + align256(8) + 4096),
            "device arena");
    uint32_t *d_in = static_cast<uint32_t *>(w.arena.take(4 * m));
    uint32_t *d_out = static_cast<uint32_t *>(w.arena.take(4 * (m + 1)));
    unsigned long long *d_tiles = static_cast<unsigned long long *>(w.arena.take(8 * 2 + 8));
    unsigned long long *d_err = static_cast<unsigned long long *>(w.arena.take(8));

    cudaStream_t s = w.stream;
    PHB_TRY(cudaMemsetAsync(d_in, 0, 4 * m, s), "memset");
    PHB_TRY(cudaMemsetAsync(d_tiles, 0, 8 * 2 + 8, s), "memset");
    PHB_TRY(cudaMemsetAsync(d_err, 0xFF, 8, s), "memset");
    ScanArgs sa{d_in, d_out, nullptr, m, d_tiles, reinterpret_cast<uint32_t *>(d_tiles + 2), 1, d_err,
                (unsigned long long)wait_ms * 1000000ull};
    PHB_TRY(launch_scan_stalled(sa, 1, s), "stalled scan");
    PHB_TRY(w.pinned.reserve(4096), "pinned");
    unsigned long long *h = static_cast<unsigned long long *>(w.pinned.data());
    PHB_TRY(cudaMemcpyAsync(h, d_err, 8, cudaMemcpyDeviceToHost, s), "D2H");
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    phobic_status st = wait_event(w.ev[7], w.timeout_ms, err);
    if (st != PHOBIC_OK) return st;
    *observed = *h == kNoError ? PHOBIC_OK : (phobic_status)(uint32_t)*h;
    return PHOBIC_OK;
}

// ------------------------------------------------------------------ query

phobic_status run_query(Worker &w, const phobic_keys *keys, const phobic_params *params, uint32_t partitions,
                        const phobic_result *built, uint32_t *positions, uint64_t *bad, std::string *err) {
    if (!keys || !params || !built || (!positions && !bad)) {
        if (err) *err = "null argument";
        return PHOBIC_ERR_INVALID;
    }
    phobic_status st = check_keys(keys, err);
    if (st != PHOBIC_OK) return st;
    const uint64_t n = keys->n;
    const uint32_t B = params->buckets;
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    PHB_TRY(w.pinned.reserve(4096), "pinned");
    unsigned long long *hword = static_cast<unsigned long long *>(w.pinned.data());
    uint64_t bytes = 8192 + align256(4 * kFulcrums) + align256(8) + align256(4 * (size_t)B * partitions) +
                     align256(4 * ((size_t)partitions + 1)) + align256(4 * n) + align256(4 * ((n + 31) / 32 + 1)) +
                     staged_bytes(keys);
    w.arena.reset();
    PHB_TRY(w.arena.reserve(bytes), "device arena");
    cudaStream_t s = w.stream;
    const void *data = keys->data;
    const uint64_t *offs = keys->offsets;
    if (!keys->on_device && n) {
        if (keys->kind == PHOBIC_KEYS_STRINGS) {
            uint64_t nb = keys->offsets[n];
            void *d = w.arena.take(nb);
            void *o = w.arena.take(8 * (n + 1));
            st = nb ? upload(w, d, keys->data, nb, s, err) : PHOBIC_OK;
            if (st == PHOBIC_OK) st = upload(w, o, keys->offsets, 8 * (n + 1), s, err);
            if (st != PHOBIC_OK) return st;
            data = d, offs = static_cast<const uint64_t *>(o);
        } else {
            void *d = w.arena.take(key_bytes(keys));
            if ((st = upload(w, d, keys->data, key_bytes(keys), s, err)) != PHOBIC_OK) return st;
            data = d;
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
        if (partitions && (st = upload(w, a, built->pilots, 4 * (size_t)B * partitions, s, err)) != PHOBIC_OK)
            return st;
        if ((st = upload(w, b, built->partition_offsets, 4 * ((size_t)partitions + 1), s, err)) != PHOBIC_OK)
            return st;
        d_pil = a, d_off = b;
    }
    PHB_TRY(cudaMemcpyAsync(hword, d_off + partitions, 4, cudaMemcpyDeviceToHost, s), "D2H n");
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    if ((st = wait_event(w.ev[7], w.timeout_ms, err)) != PHOBIC_OK) return st;
    const uint32_t n_built = (uint32_t)(*hword & 0xFFFFFFFFull);
    uint32_t *d_pos = nullptr;
    if (positions) d_pos = keys->on_device ? positions : static_cast<uint32_t *>(w.arena.take(4 * n));
    uint32_t *d_seen = nullptr;
    if (bad) {
        d_seen = static_cast<uint32_t *>(w.arena.take(4 * ((size_t)n_built / 32 + 1)));
        PHB_TRY(cudaMemsetAsync(d_seen, 0, 4 * ((size_t)n_built / 32 + 1), s), "memset");
    }
    QueryArgs qa{partitions, B, d_fulcs, d_pil, d_off, d_pos, d_seen, d_bad, n_built};
    const int grid = (int)std::min<uint64_t>((n + kMapThreads - 1) / kMapThreads, (uint64_t)w.sm_count * 8);
    if (n && partitions) PHB_TRY(launch_query(keys->kind, data, offs, n, qa, grid, s), "query");
    if (bad) PHB_TRY(cudaMemcpyAsync(hword, d_bad, 8, cudaMemcpyDeviceToHost, s), "D2H");
    if (positions && !keys->on_device && n) {
        if ((st = download(w, positions, d_pos, 4 * n, s, err)) != PHOBIC_OK) return st;
    }
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    if ((st = wait_event(w.ev[7], w.timeout_ms, err)) != PHOBIC_OK) return st;
    if (bad) *bad = *hword + (n > n_built ? n - n_built : n_built - n);
    return PHOBIC_OK;
}

}  // namespace phobicb200
