// The search's launch-shape table and the autotuner that fills it.
//
// The reference fixes its launch shapes per pipeline as specialisation constants
// (src/search_stage.cpp:36-37, include/phobicGpu/mphf_builder.h:39-45).  Here the
// shape that matters across workload sizes is how many warps search one partition
// together and how: one warp per partition when the partitions fill the GPU; for builds
// of few partitions, whose search is bound by the latency of each partition's chain of
// tries, a group of 2, 4 or 8 warps that either tries several pilot counters of one
// bucket per step (k-split: pilots per probe) or searches several small buckets at once
// and commits them in order (bucket pipeline).
//
// phobic_autotune times every shape on synthetic keys (splitmix64 on the device; three key
// sets per size, the mean of their best-of-three build times) for a ladder of partition
// counts at the caller's parameters, and records the fastest
// per (device name, P, B, partition capacity, size class) as one line of a tab-
// separated table:
//     device  partition_size  buckets  max_partition_size  max_partitions  search_group
//     search_pipeline  [build ms of each shape of kShapes...]
// A build looks its shape up in that table (the first line of its device and
// parameters whose max_partitions is >= its partition count); builds larger than
// every class, or without a line, use the partition-count rule of launch_search.
// The table is read from $PHOBIC_TUNING_FILE, else from tuning.tsv in the package
// directory beside the library (lib/..).
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "engine.hpp"
#include "kernels.cuh"

namespace phobicb200 {
namespace {

struct TuneLine {
    std::string device;
    uint32_t P, B, cap, max_parts, group, pipeline;
};

std::mutex g_tune_mu;
bool g_tune_loaded = false;
std::vector<TuneLine> g_tune;

std::string default_table_path() {
    if (const char *p = std::getenv("PHOBIC_TUNING_FILE")) return p;
    Dl_info info;
    if (dladdr(reinterpret_cast<void *>(&default_table_path), &info) && info.dli_fname) {
        std::string lib = info.dli_fname;  // <package>/lib/libphobic_b200.so
        const size_t cut = lib.rfind('/');
        if (cut != std::string::npos) {
            const std::string dir = lib.substr(0, cut);
            const size_t up = dir.rfind('/');
            return (up == std::string::npos ? std::string(".") : dir.substr(0, up)) + "/tuning.tsv";
        }
    }
    return "tuning.tsv";
}

std::vector<TuneLine> parse_lines(std::istream &f) {
    std::vector<TuneLine> out;
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::vector<std::string> col;
        std::stringstream ss(line);
        std::string c;
        while (std::getline(ss, c, '\t')) col.push_back(c);
        if (col.size() < 7) continue;
        TuneLine t;
        t.device = col[0];
        t.P = (uint32_t)std::strtoul(col[1].c_str(), nullptr, 10);
        t.B = (uint32_t)std::strtoul(col[2].c_str(), nullptr, 10);
        t.cap = (uint32_t)std::strtoul(col[3].c_str(), nullptr, 10);
        t.max_parts = (uint32_t)std::strtoul(col[4].c_str(), nullptr, 10);
        t.group = (uint32_t)std::strtoul(col[5].c_str(), nullptr, 10);
        t.pipeline = (uint32_t)std::strtoul(col[6].c_str(), nullptr, 10);
        const bool ok_group = t.group == 1 || t.group == 2 || t.group == 4 || t.group == 8;
        if (ok_group && t.pipeline <= 1) out.push_back(t);
    }
    return out;
}

std::vector<TuneLine> parse_table(const std::string &path) {
    std::ifstream f(path);
    return parse_lines(f);
}

std::vector<TuneLine> parse_table_text(const std::string &text) {
    std::istringstream f(text);
    return parse_lines(f);
}

// Whether a table line is for this device and these parameters.
bool parse_table_line_matches(const std::string &line, const std::string &dev, uint32_t P, uint32_t B, uint32_t cap) {
    const std::vector<TuneLine> one = parse_table_text(line);
    return !one.empty() && one[0].device == dev && one[0].P == P && one[0].B == B && one[0].cap == cap;
}

// Name of a device, looked up once per device: cudaGetDeviceProperties takes
// milliseconds, and a build between two of its stage events must not wait for it.
std::string device_name(int device) {
    static std::mutex mu;
    static std::vector<std::pair<int, std::string>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (const auto &e : cache)
        if (e.first == device) return e.second;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return "";
    }
    cache.emplace_back(device, prop.name);
    return prop.name;
}

// Size classes of the ladder: partition counts.
constexpr uint32_t kClasses[] = {16, 64, 256, 512, 768, 1024, 2048, 4096};
constexpr uint32_t kTuneKeySets = 3;  // key sets timed per class and shape
// The shapes the autotuner times: one warp; k-split groups of 2 and 4; bucket pipelines of
// 2, 4 and 8 warps.
constexpr SearchShape kShapes[] = {{1, false}, {2, false}, {4, false}, {2, true}, {4, true}, {8, true}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace

SearchShape choose_search_shape(const Worker &w, const phobic_params *params, uint32_t partitions) {
    if (w.search_group) return SearchShape{(int)w.search_group, w.search_pipeline != 0};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (!g_tune_loaded) {
        g_tune = parse_table(default_table_path());
        g_tune_loaded = true;
    }
    if (g_tune.empty()) return SearchShape{};
    const std::string dev = device_name(w.device);
    uint32_t cap = 0, kmax = 0;
    if (check_params(params, &cap, &kmax, nullptr) != PHOBIC_OK) return SearchShape{};
    const TuneLine *best = nullptr;
    for (const auto &t : g_tune)
        if (t.device == dev && t.P == params->partition_size && t.B == params->buckets && t.cap == cap &&
            t.max_parts >= partitions && (!best || t.max_parts < best->max_parts))
            best = &t;
    return best ? SearchShape{(int)best->group, best->pipeline != 0} : SearchShape{};
}

phobic_status autotune(Worker &w, const phobic_params *params, const char *path, uint32_t *lines_written,
                       std::string *err) {
    uint32_t cap = 0, kmax = 0;
    phobic_status st = check_params(params, &cap, &kmax, err);
    if (st != PHOBIC_OK) return st;
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    const std::string dev = device_name(w.device);
    const uint32_t P = params->partition_size, B = params->buckets;
    const uint64_t max_keys = (uint64_t)kClasses[sizeof(kClasses) / sizeof(kClasses[0]) - 1] * P;
    uint64_t *keys = nullptr;
    uint32_t *pil = nullptr, *off = nullptr;
    const uint64_t max_parts = (max_keys + P - 1) / P;
    auto cleanup = [&] {
        if (keys) cudaFree(keys);
        if (pil) cudaFree(pil);
        if (off) cudaFree(off);
        cudaGetLastError();
    };
    if (cudaMalloc(&keys, 8 * max_keys) != cudaSuccess || cudaMalloc(&pil, 4 * (size_t)B * max_parts) != cudaSuccess ||
        cudaMalloc(&off, 4 * (max_parts + 1)) != cudaSuccess) {
        cleanup();
        if (err) *err = "autotune: no device memory for the synthetic keys";
        return PHOBIC_ERR_OOM;
    }
    const uint32_t saved = w.search_group, saved_pipe = w.search_pipeline;
    std::vector<std::string> rows;
    for (uint32_t ci = 0; ci < sizeof(kClasses) / sizeof(kClasses[0]) && st == PHOBIC_OK; ci++) {
        const uint32_t parts = kClasses[ci];
        const uint64_t n = (uint64_t)parts * P;
        phobic_keys k{PHOBIC_KEYS_U64, 1, n, keys, nullptr};
        phobic_result r{1, pil, off};
        // A small build lasts as long as its slowest partition, which varies with the keys:
        // each shape is timed on kTuneKeySets key sets and scored by the sum of their times.
        double ms[kNumShapes] = {};
        for (uint32_t ks = 0; ks < kTuneKeySets && st == PHOBIC_OK; ks++) {
            if (launch_splitmix(keys, n, 0x7475ull + 97 * ci + 7919 * ks, w.stream) != cudaSuccess) {
                st = cuda_status(cudaGetLastError(), "autotune keys", err);
                break;
            }
            for (int si = 0; si < kNumShapes && st == PHOBIC_OK; si++) {
                w.search_group = (uint32_t)kShapes[si].group;
                w.search_pipeline = kShapes[si].pipeline ? 1u : 0u;
                double best = 1e30;
                for (int rep = 0; rep < 4 && st == PHOBIC_OK; rep++) {  // one warm-up, best of three
                    phobic_timings t{};
                    st = enqueue_sets(w, &k, 1, params, &r, nullptr, err);
                    if (st == PHOBIC_OK) st = finish_sets(w, nullptr, &t, err);
                    if (rep > 0 && t.total < best) best = t.total;
                }
                ms[si] += best / kTuneKeySets;
            }
        }
        if (st != PHOBIC_OK) break;
        const int win = (int)(std::min_element(ms, ms + kNumShapes) - ms);
        std::string row = dev + "\t" + std::to_string(P) + "\t" + std::to_string(B) + "\t" + std::to_string(cap) + "\t" +
                          std::to_string(parts) + "\t" + std::to_string(kShapes[win].group) + "\t" +
                          (kShapes[win].pipeline ? "1" : "0");
        for (int si = 0; si < kNumShapes; si++) {
            char t[32];
            std::snprintf(t, sizeof(t), "\t%.4f", ms[si]);
            row += t;
        }
        rows.push_back(row);
    }
    w.search_group = saved;
    w.search_pipeline = saved_pipe;
    cleanup();
    if (st != PHOBIC_OK) return st;
    const std::string out_path = path && *path ? std::string(path) : default_table_path();
    // Keep the other lines of the table (other devices and parameters), replace ours.
    std::vector<std::string> keep;
    {
        std::ifstream f(out_path);
        std::string line;
        while (std::getline(f, line)) {
            if (line.empty() || line[0] == '#') continue;
            auto parsed = parse_table_line_matches(line, dev, P, B, cap);
            if (!parsed) keep.push_back(line);
        }
    }
    // Written beside the table and renamed over it, so a reader never sees half a table.
    const std::string tmp_path = out_path + ".tmp";
    std::ofstream o(tmp_path, std::ios::trunc);
    if (!o) {
        if (err) *err = "autotune: cannot write " + tmp_path;
        return PHOBIC_ERR_INVALID;
    }
    o << "# device\tpartition_size\tbuckets\tmax_partition_size\tmax_partitions\tsearch_group\tsearch_pipeline"
         "\tbuild_ms_1\tbuild_ms_2k\tbuild_ms_4k\tbuild_ms_2p\tbuild_ms_4p\tbuild_ms_8p\n";
    for (const auto &l : keep) o << l << "\n";
    for (const auto &l : rows) o << l << "\n";
    o.close();
    if (!o || std::rename(tmp_path.c_str(), out_path.c_str()) != 0) {
        std::remove(tmp_path.c_str());
        if (err) *err = "autotune: cannot replace " + out_path;
        return PHOBIC_ERR_INVALID;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune = parse_table(out_path);
        g_tune_loaded = true;
    }
    if (lines_written) *lines_written = (uint32_t)rows.size();
    return PHOBIC_OK;
}

}  // namespace phobicb200
