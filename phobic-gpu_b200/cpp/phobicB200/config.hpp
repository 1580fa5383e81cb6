// MPHFconfig and the bucketers (reference: include/phobicGpu/mphf_config.h:16-66,
// include/phobicGpu/bucketers.h:9-50), and the initial-hash key types
// (include/phobicGpu/hasher.hpp:7-66).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "keyhash.hpp"

namespace phobicgpu {

constexpr uint32_t FULCS_INTER = 2048;

class Bucketer {
  public:
    virtual void init(double, double) {}
    virtual double getBucketRel(double relInput) const = 0;
    virtual ~Bucketer() {}
};

class UniformBucketer : public Bucketer {
  public:
    double getBucketRel(double x) const override { return x; }
};

// y(x) = (x + (1-x) ln(1-x)) (1-c) + c x with c = 0.2 lambda / sqrt(P).
class OptBucketer : public Bucketer {
  public:
    double c = 0;
    void init(double lambda, double expected_table_size) override { c = 0.2 * lambda / std::sqrt(expected_table_size); }
    double getBucketRel(double x) const override { return (x + (1.0 - x) * std::log(1.0 - x)) * (1.0 - c) + c * x; }
};

class SkewBucketer : public Bucketer {
  public:
    double getBucketRel(double x) const override { return x < 0.6 ? x / 0.6 * 0.3 : 0.3 + (x - 0.6) / 0.4 * 0.7; }
};

struct MPHFconfig {
  private:
    std::vector<uint32_t> fulcrums;

  public:
    uint32_t partitionSize;
    uint32_t bucketCountPerPartition;
    uint32_t sortingBins;
    double m_averageBucketSize;

    // B = ceil(P / lambda) with the optimized bucketer.
    MPHFconfig(double averageBucketSize = 8.0, uint32_t partition_size = 2048)
        : partitionSize(partition_size),
          bucketCountPerPartition(uint32_t(std::ceil(partition_size / averageBucketSize))),
          sortingBins(256),
          m_averageBucketSize(averageBucketSize) {
        OptBucketer b;
        setBucketer(&b);
    }

    // B = round(P / lambda) with a caller-chosen bucketer.
    MPHFconfig(Bucketer *bucketer, double averageBucketSize = 8.0, uint32_t partition_size = 2048)
        : partitionSize(partition_size),
          bucketCountPerPartition(uint32_t(std::round(partition_size / averageBucketSize))),
          sortingBins(256),
          m_averageBucketSize(averageBucketSize) {
        setBucketer(bucketer);
    }

    // Fulcrum table: 2048 samples of the bucketer curve scaled to B << 16.
    void setBucketer(Bucketer *bucketer) {
        bucketer->init(m_averageBucketSize, partitionSize);
        fulcrums.clear();
        fulcrums.push_back(0);
        const double top = double(bucketCountPerPartition << 16);
        for (size_t xi = 1; xi < FULCS_INTER - 1; xi++) {
            const double x = double(xi) / double(FULCS_INTER - 1);
            fulcrums.push_back(uint32_t(bucketer->getBucketRel(x) * top));
        }
        fulcrums.push_back(bucketCountPerPartition << 16);
    }

    const std::vector<uint32_t> &getFulcs() const { return fulcrums; }

    uint32_t partitionMaxSize() const { return partitionSize + partitionSize / 2; }
};

// ------------------------------------------------------------------ keys and initial hash

struct Key {
    uint32_t partitioner;
    uint32_t bucketer;
    uint32_t lower1;
    uint32_t lower2;

    Key() {}
    Key(uint32_t p, uint32_t b, uint32_t l1, uint32_t l2) : partitioner(p), bucketer(b), lower1(l1), lower2(l2) {}
};

// Keys that are already hashed.
struct nohash {
    static inline const Key &hash(const Key &val) { return val; }
};

// XXH3-128, seed 0: Key words are the little-endian words of (low64, high64).
struct xxhash {
    static inline Key from(phobicb200::xxh3::H128 h) {
        return Key(uint32_t(h.lo), uint32_t(h.lo >> 32), uint32_t(h.hi), uint32_t(h.hi >> 32));
    }
    static inline Key hash(const std::string &val) {
        return from(phobicb200::xxh3::hash_bytes(reinterpret_cast<const uint8_t *>(val.data()), val.size()));
    }
    static inline Key hash(uint64_t val) { return from(phobicb200::xxh3::hash_u64(val)); }
    static inline Key hash(std::pair<uint64_t, uint64_t> val) {
        return from(phobicb200::xxh3::hash_16(val.first, val.second));
    }
    static inline Key hash(const Key &val) {
        uint64_t w0 = uint64_t(val.partitioner) | (uint64_t(val.bucketer) << 32);
        uint64_t w1 = uint64_t(val.lower1) | (uint64_t(val.lower2) << 32);
        return from(phobicb200::xxh3::hash_16(w0, w1));
    }
};

}  // namespace phobicgpu
