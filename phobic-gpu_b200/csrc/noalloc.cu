// phobic_build_noalloc: the plain build for callers that cannot allocate memory.
//
// Some callers cannot call cudaMalloc: a host framework that owns the whole
// device memory pool and hands out only the buffers it sized itself, a latency-
// critical path where cudaMalloc's implicit synchronisation and driver work are
// not acceptable, or a plugin host that forbids allocation inside its callbacks.
// This entry point builds one key set with the same kernels as phobic_build, but
// takes every byte of scratch memory from one file-scope __device__ array of
// kNoAllocScratchBytes, and allocates nothing: no cudaMalloc, cudaFree,
// cudaMallocHost, no stream or event creation, no allocating library call.
// The caller passes device-resident keys and device result arrays and a stream.
//
//   * The array exists once per GPU that loads this library and stays held until
//     the process exits.
//   * Its device address is looked up once per device with cudaGetSymbolAddress
//     (host code cannot use the array's name as a device address); the first call
//     on a device does that lookup.
//   * The call is synchronous: it waits (bounded by PHOBIC_TIMEOUT_MS, default
//     120 s) for its stream and reads the status.  It copies from host memory and
//     waits on the stream, so it must not be called while that stream is being
//     captured into a CUDA graph; such a call returns PHOBIC_ERR_INVALID.
//   * Every call shares the array and it keeps the previous call's contents: the
//     counters the kernels need at zero are cleared by each call.  Calls whose
//     work would overlap on the GPU race on the array: while one call's work is
//     queued or running on a device, another call on that device returns
//     PHOBIC_ERR_BUSY.  A call that returned PHOBIC_ERR_TIMEOUT leaves its work
//     queued; calls on that device return PHOBIC_ERR_BUSY until that work has
//     drained, and the caller must synchronise the stream before it frees or
//     rewrites the keys and result arrays.
#include <atomic>
#include <cstring>
#include <mutex>

#include "engine.hpp"
#include "kernels.cuh"

namespace phobicb200 {
namespace {

// Largest build the static scratch holds.
constexpr uint64_t kNoAllocMaxKeys = 1u << 20;
constexpr uint64_t kNoAllocMaxPartitions = 1u << 16;

// Scratch layout (byte offsets, each slice 256-byte aligned).
constexpr size_t A(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffFulcs = 0;
constexpr size_t kOffDesc = kOffFulcs + A(4 * kFulcrums);
constexpr size_t kOffKeyBase = kOffDesc + A(sizeof(SetDesc));
constexpr size_t kOffPartBase = kOffKeyBase + A(16);
constexpr size_t kOffErr = kOffPartBase + A(8);
constexpr size_t kOffQueue = kOffErr + A(8);
constexpr size_t kOffCount = kOffQueue + A(64);
constexpr size_t kOffG = kOffCount + A(4 * kNoAllocMaxPartitions);
constexpr size_t kOffTiles = kOffG + A(4 * (kNoAllocMaxPartitions + 1));
constexpr size_t kTilesMax = (kNoAllocMaxPartitions + kScanTile - 1) / kScanTile;
constexpr size_t kOffLowers = kOffTiles + A(8 * kTilesMax + 8);
constexpr size_t kOffBkt = kOffLowers + A(8 * kNoAllocMaxKeys);
constexpr size_t kOffSorted = kOffBkt + A(2 * kNoAllocMaxKeys);
constexpr size_t kNoAllocScratchBytes = kOffSorted + A(8 * kNoAllocMaxKeys);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};
// 1 while a call's work may use the device's array: set when a call starts, cleared
// by a host function queued behind that call's last operation (so a call that timed
// out keeps it set until its work has really finished).
std::atomic<int> g_in_use[kMaxDevices];

void CUDART_CB release_scratch(void *device) { g_in_use[(intptr_t)device].store(0, std::memory_order_release); }

// Device address of the scratch array on the current device (looked up once).
phobic_status scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return PHOBIC_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return e == cudaErrorNoKernelImageForDevice ? PHOBIC_ERR_NO_DEVICE : PHOBIC_ERR_CUDA;
        }
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[device]);
    return PHOBIC_OK;
}

}  // namespace
}  // namespace phobicb200

using namespace phobicb200;

extern "C" phobic_status phobic_build_noalloc(const phobic_keys *keys, const phobic_params *params,
                                              const phobic_result *result, void *stream_handle) {
    std::string err;
    uint32_t cap = 0, k_max = 0;
    if (!keys || !result) return PHOBIC_ERR_INVALID;
    phobic_status st = check_params(params, &cap, &k_max, &err);
    if (st == PHOBIC_OK) st = check_keys(keys, &err);
    if (st != PHOBIC_OK) return st;
    if (!keys->on_device || !result->on_device || keys->kind == PHOBIC_KEYS_STRINGS) return PHOBIC_ERR_INVALID;
    const uint64_t n = keys->n;
    const uint32_t P = params->partition_size, B = params->buckets;
    const uint64_t m = (n + P - 1) / P;
    if (n > kNoAllocMaxKeys || m > kNoAllocMaxPartitions) return PHOBIC_ERR_BUDGET;  // beyond the static scratch
    if (!result->partition_offsets || (n && !result->pilots)) return PHOBIC_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(result->pilots) | reinterpret_cast<uintptr_t>(result->partition_offsets)) & 3)
        return PHOBIC_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream_handle);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &capture) != cudaSuccess) {
        cudaGetLastError();
        return PHOBIC_ERR_CUDA;
    }
    if (capture != cudaStreamCaptureStatusNone) return PHOBIC_ERR_INVALID;  // synchronous: not capturable

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return PHOBIC_ERR_NO_DEVICE;
    }
    unsigned char *base = nullptr;
    if ((st = scratch_address(device, &base)) != PHOBIC_OK) return st;
    int sm_count = 0;
    if (cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return PHOBIC_ERR_CUDA;
    int idle = 0;
    if (!g_in_use[device].compare_exchange_strong(idle, 1, std::memory_order_acq_rel))
        return PHOBIC_ERR_BUSY;  // another call's work may still be using the array
    const uint64_t timeout_ms = env_timeout_ms();

    uint32_t *d_fulcs = reinterpret_cast<uint32_t *>(base + kOffFulcs);
    SetDesc *d_desc = reinterpret_cast<SetDesc *>(base + kOffDesc);
    uint64_t *d_kb = reinterpret_cast<uint64_t *>(base + kOffKeyBase);
    uint32_t *d_pb = reinterpret_cast<uint32_t *>(base + kOffPartBase);
    unsigned long long *d_err = reinterpret_cast<unsigned long long *>(base + kOffErr);
    uint32_t *d_queue = reinterpret_cast<uint32_t *>(base + kOffQueue);
    uint32_t *d_count = reinterpret_cast<uint32_t *>(base + kOffCount);
    uint32_t *d_G = reinterpret_cast<uint32_t *>(base + kOffG);
    unsigned long long *d_tiles = reinterpret_cast<unsigned long long *>(base + kOffTiles);
    uint2 *d_lowers = reinterpret_cast<uint2 *>(base + kOffLowers);
    uint16_t *d_bkt = reinterpret_cast<uint16_t *>(base + kOffBkt);
    uint2 *d_sorted = reinterpret_cast<uint2 *>(base + kOffSorted);
    const uint32_t tiles = (uint32_t)((m + kScanTile - 1) / kScanTile);

    // Host-side tables live on the stack; copies from pageable memory are staged by
    // the runtime before cudaMemcpyAsync returns.
    SetDesc hd;
    std::memset(&hd, 0, sizeof(hd));
    hd.data = keys->data;
    hd.n = (uint32_t)n;
    hd.partitions = (uint32_t)m;
    hd.pilots = result->pilots;
    hd.part_off = result->partition_offsets;
    uint64_t hkb[2] = {0, n};
    uint32_t hpb[2] = {0, (uint32_t)m};

    auto cuda = [&](cudaError_t e) { return e == cudaSuccess; };
    bool ok = cuda(cudaMemcpyAsync(d_fulcs, params->fulcrums, 4 * kFulcrums, cudaMemcpyHostToDevice, s)) &&
              cuda(cudaMemcpyAsync(d_desc, &hd, sizeof(hd), cudaMemcpyHostToDevice, s)) &&
              cuda(cudaMemcpyAsync(d_kb, hkb, sizeof(hkb), cudaMemcpyHostToDevice, s)) &&
              cuda(cudaMemcpyAsync(d_pb, hpb, sizeof(hpb), cudaMemcpyHostToDevice, s)) &&
              cuda(cudaMemsetAsync(d_err, 0xFF, 8, s)) && cuda(cudaMemsetAsync(d_queue, 0, 64, s)) &&
              cuda(cudaMemsetAsync(d_count, 0, 4 * m, s)) && cuda(cudaMemsetAsync(d_tiles, 0, 8 * tiles + 8, s));
    if (ok && m == 0) ok = cuda(cudaMemsetAsync(result->partition_offsets, 0, 4, s));
    if (ok && n) {
        // The global-counter plan: one counter per partition keeps the scratch small.
        // d_count holds the counts, then (scanned in place) the placement cursors, which
        // end at the next partition's offset when both passes read the same keys.
        const uint32_t grid = (uint32_t)std::min<uint64_t>((n + kMapThreads - 1) / kMapThreads, (uint64_t)sm_count * 8);
        const MapPlan plan{false, 1, grid, 0};
        MapArgs ma{d_desc, d_kb, 1, B, n, d_fulcs, d_count, nullptr, nullptr, d_lowers, d_bkt, d_err,
                   (uint32_t)m, 1, 0};
        ScanArgs sa{d_count, d_G, d_count, (uint32_t)m, d_tiles, reinterpret_cast<uint32_t *>(d_tiles + tiles), 1,
                    d_err, 0};
        SearchArgs qa{d_desc, d_pb, 1, (uint32_t)m, d_G, 1, d_lowers, d_bkt, d_sorted, nullptr, B, cap, k_max,
                      d_queue, d_err, d_count};
        uint64_t kc_index = 0, kc_mask = 0;
        ok = cuda(launch_map_count(keys->kind, ma, plan, s));
        if (ok && take_key_change(n, keys->kind, &kc_index, &kc_mask))
            ok = cuda(launch_change_key(const_cast<void *>(keys->data), kc_index, kc_mask, s));
        ok = ok && cuda(launch_scan(sa, s)) &&
             cuda(launch_check_sizes(d_G, (uint32_t)m, 1, cap, d_pb, 1, d_err, nullptr, s)) &&
             cuda(launch_scatter(keys->kind, ma, plan, s)) && cuda(launch_search(qa, sm_count, s));
    }
    if (!ok) cudaGetLastError();
    // Bounded wait for everything queued above (also after a failed launch: work queued
    // before it may still use the array).
    st = wait_stream(s, timeout_ms, &err);
    if (st == PHOBIC_ERR_TIMEOUT) {
        // The work keeps the array until it drains: release it from the stream then (if
        // even that cannot be queued, the array stays taken and later calls get BUSY).
        if (cudaLaunchHostFunc(s, release_scratch, (void *)(intptr_t)device) != cudaSuccess) cudaGetLastError();
        return st;
    }
    unsigned long long word = kNoError;
    // The stream is idle: this copy to pageable memory returns at once.
    if (st == PHOBIC_OK && ok) ok = cuda(cudaMemcpyAsync(&word, d_err, 8, cudaMemcpyDeviceToHost, s)) &&
                                    cuda(cudaStreamSynchronize(s));
    if (!ok) cudaGetLastError();
    g_in_use[device].store(0, std::memory_order_release);
    if (st != PHOBIC_OK) return st;
    if (!ok) return PHOBIC_ERR_CUDA;
    return word == kNoError ? PHOBIC_OK : (phobic_status)(uint32_t)word;
}

extern "C" phobic_status phobic_debug_change_key(uint64_t index, uint64_t xor_mask) {
    set_key_change(index, xor_mask);
    return PHOBIC_OK;
}
