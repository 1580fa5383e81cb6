// The MPHF container and query (reference: include/phobicGpu/mphf.hpp:20-97).
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "config.hpp"
#include "encoders.hpp"

namespace phobicgpu {

// Writes serialised fields in visit order: a trivially copyable value as its bytes,
// a vector as its size_t count followed by its elements.
struct ByteSaver {
    std::vector<uint8_t> out;
    void put(const void *p, size_t n) {
        const uint8_t *b = static_cast<const uint8_t *>(p);
        out.insert(out.end(), b, b + n);
    }
    template <typename T>
    void visit(std::vector<T> &v) {
        size_t n = v.size();
        put(&n, sizeof(n));
        if constexpr (std::is_trivially_copyable_v<T>) {
            if (n) put(v.data(), n * sizeof(T));
        } else {
            for (auto &e : v) visit(e);
        }
    }
    template <typename T>
    void visit(T &v) {
        if constexpr (std::is_trivially_copyable_v<T>) put(&v, sizeof(T));
        else v.visit(*this);
    }
};

// Reads serialised fields in visit order: a trivially copyable value as its bytes,
// a vector as its size_t count followed by its elements.
struct ByteLoader {
    const uint8_t *bytes;
    size_t size;
    size_t pos = 0;
    bool ok = true;

    void get(void *dst, size_t n) {
        if (!ok || n > size - pos) {
            ok = false;
            std::memset(dst, 0, n);
            return;
        }
        std::memcpy(dst, bytes + pos, n);
        pos += n;
    }
    template <typename T>
    void visit(std::vector<T> &v) {
        size_t n = 0;
        get(&n, sizeof(n));
        if (!ok) return;
        if constexpr (std::is_trivially_copyable_v<T>) {
            if (n > (size - pos) / sizeof(T)) {
                ok = false;
                return;
            }
            v.resize(n);
            if (n) get(v.data(), n * sizeof(T));
        } else {
            v.resize(n);
            for (auto &e : v) visit(e);
        }
    }
    template <typename T>
    void visit(T &v) {
        if constexpr (std::is_trivially_copyable_v<T>) get(&v, sizeof(T));
        else v.visit(*this);
    }
};

template <typename PilotEncoder, typename PartitionOffsetEncoder, typename Hasher>
class MPHF {
  private:
    std::vector<uint32_t> fulcs;
    uint32_t partitions = 0;
    PilotEncoder pilots;
    PartitionOffsetEncoder partitionOffsets;

    // Bucket by the 64-bit fulcrum interpolation (mphf.hpp:42-49).
    uint64_t getBucket(uint32_t bucketer) const { return phobicb200::bucket_of_query(bucketer, fulcs.data()); }

  public:
    using pilot_encoder_type = PilotEncoder;
    using offset_encoder_type = PartitionOffsetEncoder;

    PilotEncoder &getPilotEncoder() { return pilots; }
    PartitionOffsetEncoder &getPartitionOffsetEncoder() { return partitionOffsets; }
    uint32_t getPartitions() const { return partitions; }

    constexpr static bool noHash() { return std::is_same_v<Hasher, nohash>; }

    template <typename keyType>
    static inline Key initialHash(const keyType &keyRaw) {
        return Hasher::hash(keyRaw);
    }

    // Encodes the serialized pilot layout: pilots[b * partitions + p] and the
    // exclusive partition offsets [partitions + 1] (mphf.hpp:65-75).
    void setData(const std::vector<uint32_t> &pilot_values, std::vector<uint32_t> &offsets, uint32_t parts,
                 MPHFconfig config) {
        fulcs = config.getFulcs();
        partitions = parts;
        partitionOffsets.encode(offsets.begin(), config.partitionSize, parts + 1);
        pilots.encode(pilot_values.begin(), parts, config.bucketCountPerPartition);  // columns in parallel
    }

    // The state setData produces, read back from the encoders' serialised bytes
    // (pilot encoder, then partition-offset encoder, in visit order, as
    // phobic_encode and phobic_encode_gpu write them).  False when the bytes do
    // not hold exactly the two encoders.
    bool loadEncoded(const uint8_t *bytes, size_t size, uint32_t parts, const MPHFconfig &config) {
        fulcs = config.getFulcs();
        partitions = parts;
        pilots.set_shape(parts, config.bucketCountPerPartition);
        partitionOffsets.set_shape(config.partitionSize);
        ByteLoader loader{bytes, size};
        pilots.visit(loader);
        partitionOffsets.visit(loader);
        return loader.ok && loader.pos == size;
    }

    // The whole function as bytes, in visit order: partition count, fulcrum table,
    // pilot encoder, partition-offset encoder (vectors as a size_t count followed
    // by their elements).
    std::vector<uint8_t> save() {
        ByteSaver saver;
        visit(saver);
        return std::move(saver.out);
    }

    // The function saved by save().  The bytes hold everything but the partition
    // size, which the offset encoder's expected-offset line needs; the bucket count
    // per partition is the last fulcrum >> 16 (mphf_config.h:44-55).  False when the
    // bytes are not one saved function.
    bool load(const uint8_t *bytes, size_t size, uint32_t partition_size) {
        ByteLoader loader{bytes, size};
        loader.visit(partitions);
        loader.visit(fulcs);
        if (!loader.ok || fulcs.size() != phobicb200::kFulcrums) return false;
        pilots.set_shape(partitions, fulcs.back() >> 16);
        partitionOffsets.set_shape(partition_size);
        pilots.visit(loader);
        partitionOffsets.visit(loader);
        return loader.ok && loader.pos == size;
    }

    // Slot of a key in [0, n) (mphf.hpp:77-86).
    template <typename keyType>
    inline uint32_t operator()(const keyType &keyRaw) const {
        const Key key = initialHash(keyRaw);
        const uint64_t partition = (uint64_t(key.partitioner) * uint64_t(partitions)) >> 32;
        const uint64_t bucket = getBucket(key.bucketer);
        const uint32_t pilot = uint32_t(pilots.access(partition, bucket));
        const uint32_t offset = uint32_t(partitionOffsets.access(partition));
        const uint32_t size = uint32_t(partitionOffsets.access(partition + 1)) - offset;
        return offset + phobicb200::slot_of(pilot, key.lower1, key.lower2, size);
    }

    float getBitsPerKey() const {
        return float(pilots.num_bits() + partitionOffsets.num_bits() + 32 * fulcs.size() + 32 * partitions) /
               float(partitionOffsets.access(partitions));
    }

    std::string getResultLine() {
        const double n = float(partitionOffsets.access(partitions));
        return "total_bits=" + std::to_string(getBitsPerKey()) + " pilot_bits=" + std::to_string(pilots.num_bits() / n) +
               " offsets_bits=" + std::to_string(partitionOffsets.num_bits() / n);
    }

    // Serialisation of the whole function (the reference's MPHF has none): the
    // partition count, the fulcrum table, then the two encoders in their own
    // visit order.
    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(partitions);
        visitor.visit(fulcs);
        pilots.visit(visitor);
        partitionOffsets.visit(visitor);
    }
};

}  // namespace phobicgpu
