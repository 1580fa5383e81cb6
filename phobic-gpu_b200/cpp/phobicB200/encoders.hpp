// Pilot and partition-offset encoders: the host end of the construction path.
//
// The B200 build hands the encoders two arrays (bucket-major pilots and the
// exclusive partition offsets) exactly as the reference does through
// Mphf::setData (include/phobicGpu/mphf.hpp:65-75).  These encoders keep the
// reference's type names and formats (include/encoders/**):
//   base:       compact, dictionary, rice, elias_fano, sdc
//   pilots:     interleaved_encoder<E> (one E per bucket index over all partitions),
//               interleaved_encoder_dual<E1, E2>, mono_encoder<E>
//   offsets:    diff_partition_encoder<E> (zig-zag difference to i*P),
//               direct_partition_encoder<E>
// so an MPHF serialised with visit() has the same bytes as the reference's.
#pragma once

#include <cstdint>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "succinct.hpp"

namespace phobicgpu {

// ------------------------------------------------------------------ base encoders

struct compact {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) { m_values.build(begin, n); }
    static std::string name() { return "compact"; }
    size_t size() const { return m_values.size(); }
    size_t num_bits() const { return m_values.bytes() * 8; }
    uint64_t access(uint64_t i) const { return m_values.access(i); }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(m_values); }

  private:
    compact_vector m_values;
};

struct rice {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) { m_values.encode(begin, n); }
    static std::string name() { return "rice"; }
    size_t size() const { return m_values.size(); }
    size_t num_bits() const { return m_values.bytes() * 8; }
    uint64_t access(uint64_t i) const { return m_values.access(i); }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(m_values); }

  private:
    rice_sequence m_values;
};

// Dictionary codes: every distinct value gets a rank by non-increasing frequency
// (encoders.hpp:145-177).  Ranks of equal frequency depend on the standard
// library's hash-table iteration order and on std::sort; the same standard
// library reproduces the reference's bytes.
namespace dict_detail {
template <typename Iterator>
std::pair<std::vector<uint64_t>, std::vector<uint64_t>> ranks_and_dictionary(Iterator begin, uint64_t n) {
    std::unordered_map<uint64_t, uint64_t> freq;
    for (Iterator it = begin, end = begin + n; it != end; ++it) {
        auto f = freq.find(*it);
        if (f != freq.end()) f->second += 1;
        else freq[*it] = 1;
    }
    std::vector<std::pair<uint64_t, uint64_t>> by_freq;
    by_freq.reserve(freq.size());
    for (auto kv : freq) by_freq.emplace_back(kv.first, kv.second);
    std::sort(by_freq.begin(), by_freq.end(), [](auto const &a, auto const &b) { return a.second > b.second; });
    freq.clear();
    std::vector<uint64_t> dict;
    dict.reserve(freq.size());
    for (uint64_t i = 0; i != by_freq.size(); ++i) {
        freq.insert({by_freq[i].first, i});
        dict.push_back(by_freq[i].first);
    }
    std::vector<uint64_t> ranks;
    ranks.reserve(n);
    for (Iterator it = begin, end = begin + n; it != end; ++it) ranks.push_back(freq[*it]);
    return {ranks, dict};
}
}  // namespace dict_detail

struct dictionary {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) {
        auto rd = dict_detail::ranks_and_dictionary(begin, n);
        m_ranks.build(rd.first.begin(), rd.first.size());
        m_dict.build(rd.second.begin(), rd.second.size());
    }
    static std::string name() { return "dictionary"; }
    size_t size() const { return m_ranks.size(); }
    size_t num_bits() const { return (m_ranks.bytes() + m_dict.bytes()) * 8; }
    uint64_t access(uint64_t i) const { return m_dict.access(m_ranks.access(i)); }
    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_ranks);
        visitor.visit(m_dict);
    }

  private:
    compact_vector m_ranks;
    compact_vector m_dict;
};

struct elias_fano {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) { m_values.encode(begin, n); }
    static std::string name() { return "elias_fano"; }
    size_t size() const { return m_values.size(); }
    size_t num_bits() const { return m_values.num_bits(); }
    uint64_t access(uint64_t i) const { return m_values.diff(i); }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(m_values); }

  private:
    ef_sequence<true> m_values;
};

struct sdc {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) {
        auto rd = dict_detail::ranks_and_dictionary(begin, n);
        m_ranks.build(rd.first.begin(), rd.first.size());
        m_dict.build(rd.second.begin(), rd.second.size());
    }
    static std::string name() { return "sdc"; }
    size_t size() const { return m_ranks.size(); }
    size_t num_bits() const { return (m_ranks.bytes() + m_dict.bytes()) * 8; }
    uint64_t access(uint64_t i) const { return m_dict.access(m_ranks.access(i)); }
    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_ranks);
        visitor.visit(m_dict);
    }

  private:
    sdc_sequence m_ranks;
    compact_vector m_dict;
};

// ------------------------------------------------------------------ pilot encoders

// One base encoder per bucket index, each over the `partitions` pilots of that
// column of the bucket-major layout (interleaved_encoder.hpp:8-15).
template <typename BaseEncoder>
struct interleaved_encoder {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t partitions, uint64_t buckets) {
        encoders.resize(buckets);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t j = 0; j < (int64_t)buckets; j++) encoders[j].encode(begin + j * partitions, partitions);
    }
    uint64_t access(uint64_t partition, uint64_t bucket) const { return encoders[bucket].access(partition); }
    // Shape for loading from serialised bytes (the bytes do not hold the column count).
    void set_shape(uint64_t, uint64_t buckets) { encoders.assign(buckets, BaseEncoder()); }
    std::string name() { return "InterEncoder<" + BaseEncoder::name() + ">"; }
    uint64_t num_bits() const {
        uint64_t s = 0;
        for (auto &e : encoders) s += e.num_bits();
        return s;
    }
    template <typename Visitor>
    void visit(Visitor &visitor) {
        for (auto &e : encoders) e.visit(visitor);
    }

  private:
    std::vector<BaseEncoder> encoders;
};

// The first floor(buckets * tradeoff) columns with Enc1, the rest with Enc2
// (interleaved_encoder_dual.hpp:10-18).
template <typename BaseEncoder1, typename BaseEncoder2>
struct interleaved_encoder_dual {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t partitions, uint64_t buckets) {
        initialized = true;
        buckets1 = buckets * tradeoff;
        encoder1.encode(begin, partitions, buckets1);
        encoder2.encode(begin + buckets1 * partitions, partitions, buckets - buckets1);
    }
    void setEncoderTradeoff(float enc_tradeoff) { tradeoff = enc_tradeoff; }
    uint64_t access(uint64_t partition, uint64_t bucket) const {
        return bucket < buckets1 ? encoder1.access(partition, bucket) : encoder2.access(partition, bucket - buckets1);
    }
    std::string name() {
        return "InterEncoderDual<" + BaseEncoder1::name() + "," + BaseEncoder2::name() + "," + std::to_string(tradeoff) +
               ">";
    }
    uint64_t num_bits() const { return encoder1.num_bits() + encoder2.num_bits(); }
    template <typename Visitor>
    void visit(Visitor &visitor) {
        encoder1.visit(visitor);
        encoder2.visit(visitor);
    }

  private:
    bool initialized = false;
    uint64_t buckets1 = 0;
    float tradeoff = 0.5;
    interleaved_encoder<BaseEncoder1> encoder1;
    interleaved_encoder<BaseEncoder2> encoder2;
};

// All pilots as one sequence, bucket-major (mono_encoders.hpp:15-33).
template <typename BaseEncoder>
struct mono_encoder {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t partitions_, uint64_t buckets) {
        partitions = partitions_;
        enc.encode(begin, partitions * buckets);
    }
    std::string name() { return BaseEncoder::name(); }
    size_t size() const { return enc.size(); }
    size_t num_bits() const { return enc.num_bits(); }
    uint64_t access(uint64_t partition, uint64_t bucket) const { return enc.access(partitions * bucket + partition); }
    void set_shape(uint64_t partitions_, uint64_t) { partitions = partitions_; }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(enc); }

  private:
    uint64_t partitions = 0;
    BaseEncoder enc;
};

// ------------------------------------------------------------------ partition-offset encoders

// Value i stored as the zig-zag-like code (|v - i*P| << 1) | (v - i*P > 0)
// (linear_diff_encoder.hpp:15-28).
template <typename BaseEncoder>
struct linear_diff_encoder {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t size, uint64_t inc) {
        increment = int64_t(inc);
        std::vector<uint64_t> codes;
        codes.reserve(size);
        int64_t expected = 0;
        for (uint64_t i = 0; i != size; ++i, ++begin) {
            const int64_t d = int64_t(*begin) - expected;
            const uint64_t a = uint64_t(d < 0 ? -d : d);
            codes.push_back((a << 1) | uint64_t(d > 0));
            expected += increment;
        }
        enc.encode(codes.begin(), size);
    }
    static std::string name() { return BaseEncoder::name(); }
    size_t size() const { return enc.size(); }
    size_t num_bits() const { return enc.num_bits(); }
    void set_increment(uint64_t inc) { increment = int64_t(inc); }
    uint64_t access(uint64_t i) const {
        const uint64_t c = enc.access(i);
        const int64_t d = (int64_t(c & 1) * 2 - 1) * int64_t(c >> 1);
        return uint64_t(d + int64_t(i * increment));
    }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(enc); }

  private:
    int64_t increment = 0;
    BaseEncoder enc;
};

template <typename BaseEncoder>
struct diff_partition_encoder {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t partition_size, uint64_t count) { enc.encode(begin, count, partition_size); }
    static std::string name() { return "DiffToExpected<" + BaseEncoder::name() + ">"; }
    void set_shape(uint64_t partition_size) { enc.set_increment(partition_size); }
    size_t size() const { return enc.size(); }
    size_t num_bits() const { return enc.num_bits(); }
    uint64_t access(uint64_t partition) const { return enc.access(partition); }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(enc); }

  private:
    linear_diff_encoder<BaseEncoder> enc;
};

template <typename BaseEncoder>
struct direct_partition_encoder {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t, uint64_t count) { enc.encode(begin, count); }
    static std::string name() { return "Direct<" + BaseEncoder::name() + ">"; }
    void set_shape(uint64_t) {}
    size_t size() const { return enc.size(); }
    size_t num_bits() const { return enc.num_bits(); }
    uint64_t access(uint64_t partition) const { return enc.access(partition); }
    template <typename Visitor>
    void visit(Visitor &visitor) { visitor.visit(enc); }

  private:
    BaseEncoder enc;
};

// Encoder codes of phobic_encode / phobic_encode_gpu for the encoders whose bytes
// the GPU writes (compact-vector encoders); -1 for the others.
template <typename E>
struct gpu_pilot_code { static constexpr int value = -1; };
template <>
struct gpu_pilot_code<interleaved_encoder<compact>> { static constexpr int value = 0; };
template <>
struct gpu_pilot_code<mono_encoder<compact>> { static constexpr int value = 3; };
template <typename E>
struct gpu_offset_code { static constexpr int value = -1; };
template <>
struct gpu_offset_code<diff_partition_encoder<compact>> { static constexpr int value = 0; };
template <>
struct gpu_offset_code<direct_partition_encoder<compact>> { static constexpr int value = 1; };

}  // namespace phobicgpu
