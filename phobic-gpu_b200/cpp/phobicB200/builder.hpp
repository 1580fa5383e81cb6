// MPHFbuilder: builds an MPHF through the B200 engine (C ABI, include/phobic_b200.h).
//
// Same surface as the reference's builder (include/phobicGpu/mphf_builder.h:18-49,
// 315-321): MPHFbuilder(MPHFconfig), HostTimer build(const std::vector<keyType>&, Mphf&),
// for keyType in {uint64_t, std::string, std::pair<uint64_t,uint64_t>, Key}.  The host
// hash, the Vulkan runtime and the seven compute stages are replaced by one call to
// phobic_build, which hashes on the device and returns the pilots and partition
// offsets that Mphf::setData encodes.  For the compact-vector encoders the result
// stays on the device and phobic_encode_gpu writes the encoders' bytes, which the
// MPHF loads.  Link with -lphobic_b200.
#pragma once

#include <chrono>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "config.hpp"
#include "encoders.hpp"
#include "phobic_b200.h"

namespace phobicgpu {

// Wall-clock labels in the style of the reference's HostTimer (include/app/host_timer.h).
class HostTimer {
  public:
    HostTimer() : start_(std::chrono::steady_clock::now()), last_(start_) {}

    double elapsed() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start_).count();
    }
    void addLabel(const std::string &name) {
        auto now = std::chrono::steady_clock::now();
        labels_.push_back({name, std::chrono::duration<double, std::milli>(now - last_).count()});
        last_ = now;
    }
    void addLabelManually(const std::string &name, double ms) { labels_.push_back({name, ms}); }
    const std::vector<std::pair<std::string, double>> &labels() const { return labels_; }

    // "label=<ns per key> " for every label (benchmark.cpp:81-90 RESULT style).
    std::string getResultStyle(size_t n) const {
        std::string out;
        for (auto &l : labels_) out += l.first + "=" + std::to_string(l.second * 1e6 / double(n ? n : 1)) + " ";
        return out;
    }
    void printLabels(size_t n) const {
        for (auto &l : labels_) std::cout << l.first << ": " << l.second << " ms, " << l.second * 1e6 / double(n ? n : 1)
                                          << " ns/key" << std::endl;
    }

  private:
    std::chrono::steady_clock::time_point start_, last_;
    std::vector<std::pair<std::string, double>> labels_;
};

class MPHFbuilder {
  public:
    explicit MPHFbuilder(MPHFconfig config = MPHFconfig(), int device = 0) : config_(std::move(config)) {
        phobic_status s = phobic_ctx_create(device, &ctx_);
        if (s != PHOBIC_OK) throw std::runtime_error(std::string("phobic: ") + phobic_status_string(s));
    }
    ~MPHFbuilder() {
        if (ctx_) phobic_ctx_destroy(ctx_);
    }
    MPHFbuilder(const MPHFbuilder &) = delete;
    MPHFbuilder &operator=(const MPHFbuilder &) = delete;

    const MPHFconfig &config() const { return config_; }
    phobic_ctx *context() { return ctx_; }

    template <typename Mphf, typename keyType>
    HostTimer build(const std::vector<keyType> &keys, Mphf &f) {
        HostTimer timer;
        phobic_params params;
        std::memset(&params, 0, sizeof(params));
        params.partition_size = config_.partitionSize;
        params.buckets = config_.bucketCountPerPartition;
        const std::vector<uint32_t> &fulcs = config_.getFulcs();
        std::memcpy(params.fulcrums, fulcs.data(), sizeof(params.fulcrums));

        phobic_keys k{};
        std::vector<uint8_t> bytes;
        std::vector<uint64_t> offsets;
        if constexpr (std::is_same_v<keyType, uint64_t>) {
            k = phobic_keys{PHOBIC_KEYS_U64, 0, keys.size(), keys.data(), nullptr};
        } else if constexpr (std::is_same_v<keyType, std::string>) {
            offsets.resize(keys.size() + 1, 0);
            for (size_t i = 0; i < keys.size(); i++) offsets[i + 1] = offsets[i] + keys[i].size();
            bytes.resize(offsets.back());
            for (size_t i = 0; i < keys.size(); i++)
                if (!keys[i].empty()) std::memcpy(bytes.data() + offsets[i], keys[i].data(), keys[i].size());
            k = phobic_keys{PHOBIC_KEYS_STRINGS, 0, keys.size(), bytes.data(), offsets.data()};
        } else {
            static_assert(sizeof(keyType) == 16, "keys must be uint64_t, std::string, pair<u64,u64> or Key");
            k = phobic_keys{Mphf::noHash() ? PHOBIC_KEYS_PREHASHED : PHOBIC_KEYS_BYTES16, 0, keys.size(), keys.data(),
                            nullptr};
        }
        timer.addLabel("input_pack");
        const uint32_t partitions = phobic_partitions(keys.size(), config_.partitionSize);
        constexpr int pe = gpu_pilot_code<typename Mphf::pilot_encoder_type>::value;
        constexpr int oe = gpu_offset_code<typename Mphf::offset_encoder_type>::value;
        if constexpr (pe >= 0 && oe >= 0) {
            // Compact-vector encoders: the result stays on the device and is encoded
            // there; only the encoded bytes come back.
            phobic_result r{};
            phobic_timings t{};
            check(phobic_ctx_result(ctx_, config_.bucketCountPerPartition, partitions, &r));
            check(phobic_build(ctx_, &k, &params, &r, &t));
            timer.addLabel("gpu_build");
            add_gpu_labels(timer, t);
            size_t size = 0;
            check(phobic_encode_gpu(ctx_, pe, oe, &r, partitions, &params, nullptr, 0, 0, &size, nullptr));
            std::vector<uint8_t> encoded(size);
            check(phobic_encode_gpu(ctx_, pe, oe, &r, partitions, &params, encoded.data(), size, 0, &size, nullptr));
            if (!f.loadEncoded(encoded.data(), size, partitions, config_))
                throw std::runtime_error("phobic: encoded bytes do not match the MPHF's encoders");
            timer.addLabel("encoding");
            return timer;
        }
        std::vector<uint32_t> pilots((size_t)partitions * config_.bucketCountPerPartition);
        std::vector<uint32_t> part_off(partitions + 1);
        phobic_result r{0, pilots.data(), part_off.data()};
        phobic_timings t{};
        check(phobic_build(ctx_, &k, &params, &r, &t));
        timer.addLabel("gpu_build");
        add_gpu_labels(timer, t);
        f.setData(pilots, part_off, partitions, config_);
        timer.addLabel("encoding");
        return timer;
    }

  private:
    void check(phobic_status s) const {
        if (s != PHOBIC_OK) throw std::runtime_error(std::string("phobic: ") + phobic_last_error(ctx_));
    }
    static void add_gpu_labels(HostTimer &timer, const phobic_timings &t) {
        timer.addLabelManually("GPU_input_transfer", t.input_transfer);
        timer.addLabelManually("GPU_bucket_sizes", t.bucket_sizes);
        timer.addLabelManually("GPU_partition_offsets", t.partition_offsets);
        timer.addLabelManually("GPU_key_redistribution", t.key_redistribution);
        timer.addLabelManually("GPU_search", t.search);
        timer.addLabelManually("GPU_result_transfer", t.result_transfer);
    }

    MPHFconfig config_;
    phobic_ctx *ctx_ = nullptr;
};

}  // namespace phobicgpu
