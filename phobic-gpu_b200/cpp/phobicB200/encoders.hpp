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

#include <algorithm>
#include <cstdint>
#include <memory>
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
// (encoders.hpp:145-177).  Ranks of equal frequency follow the standard library's
// hash-table iteration order and std::sort, as in the reference.
//
// The reference counts with find/insert on a std::unordered_map for every value
// and looks every value up again for its rank.  Here the counting and the rank
// lookups use a flat open-addressing table, and the std::unordered_map only
// receives the distinct values, in first-occurrence order, with operator[]: the
// reference's map changes only when a value is first seen, so the same insertions
// in the same order give the same buckets, the same node order and therefore the
// same iteration order (node memory comes from a per-call arena, which the order
// does not depend on).  std::sort then sees the same sequence and returns the
// same permutation, so the bytes are the reference's.
namespace dict_detail {

// Value -> u64 slot value; open addressing with linear probing, grown at half load.
class FlatMap {
  public:
    explicit FlatMap(size_t expect) {
        int lg = 4;
        while ((size_t(1) << lg) < 2 * expect && lg < 40) lg++;
        init(lg);
    }
    // Slot of v, inserted with value 0 when absent (*fresh says which).  A slot
    // index is valid until the next insertion.
    size_t find_or_insert(uint64_t v, bool *fresh) {
        if (2 * (used_ + 1) > keys_.size()) grow();
        size_t h = home(v);
        while (full_[h]) {
            if (keys_[h] == v) {
                *fresh = false;
                return h;
            }
            h = (h + 1) & mask_;
        }
        full_[h] = 1;
        keys_[h] = v;
        vals_[h] = 0;
        used_++;
        *fresh = true;
        return h;
    }
    // Slot of a value known to be present.
    size_t find(uint64_t v) const {
        size_t h = home(v);
        while (keys_[h] != v || !full_[h]) h = (h + 1) & mask_;
        return h;
    }
    uint64_t &value(size_t slot) { return vals_[slot]; }

  private:
    void init(int lg) {
        shift_ = 64 - lg;
        mask_ = (size_t(1) << lg) - 1;
        keys_.assign(size_t(1) << lg, 0);
        vals_.assign(size_t(1) << lg, 0);
        full_.assign(size_t(1) << lg, 0);
        used_ = 0;
    }
    size_t home(uint64_t v) const { return size_t((v * 0x9E3779B97F4A7C15ull) >> shift_); }
    void grow() {
        std::vector<uint64_t> k, v;
        std::vector<uint8_t> f;
        k.swap(keys_), v.swap(vals_), f.swap(full_);
        init(64 - shift_ + 1);
        for (size_t i = 0; i < k.size(); i++) {
            if (!f[i]) continue;
            size_t h = home(k[i]);
            while (full_[h]) h = (h + 1) & mask_;
            full_[h] = 1, keys_[h] = k[i], vals_[h] = v[i];
            used_++;
        }
    }
    std::vector<uint64_t> keys_, vals_;
    std::vector<uint8_t> full_;
    size_t mask_ = 0, used_ = 0;
    int shift_ = 64;
};

// Bump allocation for one call's hash-map nodes and bucket arrays; released with the arena.
class NodeArena {
  public:
    void *take(size_t bytes, size_t align) {
        size_t at = (used_ + align - 1) & ~(align - 1);
        if (blocks_.empty() || at + bytes > cap_) {
            cap_ = std::max<size_t>(size_t(1) << 20, bytes + align);
            blocks_.emplace_back(new char[cap_]);
            used_ = 0;
            at = (reinterpret_cast<uintptr_t>(blocks_.back().get()) % align)
                     ? align - reinterpret_cast<uintptr_t>(blocks_.back().get()) % align
                     : 0;
        }
        used_ = at + bytes;
        return blocks_.back().get() + at;
    }

  private:
    std::vector<std::unique_ptr<char[]>> blocks_;
    size_t used_ = 0, cap_ = 0;
};

template <typename T>
struct ArenaAlloc {
    using value_type = T;
    NodeArena *arena;
    explicit ArenaAlloc(NodeArena *a) : arena(a) {}
    template <typename U>
    ArenaAlloc(const ArenaAlloc<U> &o) : arena(o.arena) {}
    T *allocate(size_t n) { return static_cast<T *>(arena->take(n * sizeof(T), alignof(T))); }
    void deallocate(T *, size_t) {}
    template <typename U>
    bool operator==(const ArenaAlloc<U> &o) const { return arena == o.arena; }
    template <typename U>
    bool operator!=(const ArenaAlloc<U> &o) const { return arena != o.arena; }
};

template <typename Iterator>
std::pair<std::vector<uint64_t>, std::vector<uint64_t>> ranks_and_dictionary(Iterator begin, uint64_t n) {
    // Counts, and the distinct values in first-occurrence order.
    FlatMap counts(std::min<uint64_t>(n, 1u << 16));
    std::vector<uint64_t> first_seen;
    for (Iterator it = begin, end = begin + n; it != end; ++it) {
        bool fresh;
        const size_t s = counts.find_or_insert(uint64_t(*it), &fresh);
        if (fresh) first_seen.push_back(uint64_t(*it));
        counts.value(s) += 1;
    }
    // The reference's map, built by the same operator[] insertions in the same order.
    NodeArena arena;
    using Map = std::unordered_map<uint64_t, uint64_t, std::hash<uint64_t>, std::equal_to<uint64_t>,
                                   ArenaAlloc<std::pair<const uint64_t, uint64_t>>>;
    Map freq{ArenaAlloc<std::pair<const uint64_t, uint64_t>>(&arena)};
    for (uint64_t v : first_seen) freq[v] = 1;
    std::vector<std::pair<uint64_t, uint64_t>> by_freq;
    by_freq.reserve(freq.size());
    for (auto kv : freq) by_freq.emplace_back(kv.first, counts.value(counts.find(kv.first)));
    std::sort(by_freq.begin(), by_freq.end(), [](auto const &a, auto const &b) { return a.second > b.second; });
    std::vector<uint64_t> dict;
    dict.reserve(by_freq.size());
    for (uint64_t i = 0; i != by_freq.size(); ++i) {
        counts.value(counts.find(by_freq[i].first)) = i;  // the value's rank from here on
        dict.push_back(by_freq[i].first);
    }
    std::vector<uint64_t> ranks;
    ranks.reserve(n);
    for (Iterator it = begin, end = begin + n; it != end; ++it) ranks.push_back(counts.value(counts.find(uint64_t(*it))));
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
