// Succinct building blocks of the pilot and partition-offset encoders.
//
// These are the storage formats of the reference's encoders
// (include/encoders/base/{bit_vector,compact_vector,darray,rice_sequence,
// ef_sequence,sdc_sequence}.hpp, themselves PTHash's formats).  The bit layout
// and the member order of visit() are kept, so an encoder built here serialises
// to the same bytes as the reference's on the same input.  Helper names follow
// the reference where user code can see them (bit_vector, compact_vector,
// darray1, rice_sequence, ef_sequence, sdc_sequence).
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace phobicgpu {

namespace bits {

inline uint64_t words_for(uint64_t nbits) { return (nbits + 63) / 64; }

template <typename T>
inline size_t vec_bytes(const std::vector<T> &v) { return sizeof(T) * v.size() + sizeof(size_t); }

// Index of the highest set bit (x != 0).
inline uint64_t msb(uint64_t x) { return 63 - (uint64_t)__builtin_clzll(x); }

// Number of bits needed to write x: 0 -> 1 (a width of 0 is never used).
inline uint64_t width_for(uint64_t max_value) { return max_value ? msb(max_value) + 1 : 1; }

// Position of the k-th set bit of x (k < popcount(x)).
inline uint64_t select_in_word(uint64_t x, uint64_t k) {
    for (uint64_t i = 0; i < k; i++) x &= x - 1;
    return (uint64_t)__builtin_ctzll(x);
}

}  // namespace bits

// Growable bit array written LSB first into 64-bit words.
class bit_vector_builder {
  public:
    explicit bit_vector_builder(uint64_t size = 0) : m_size(size), m_words(bits::words_for(size), 0) {}

    void push_back(bool b) {
        if ((m_size & 63) == 0) m_words.push_back(0);
        m_words.back() |= uint64_t(b) << (m_size & 63);
        m_size++;
    }
    void set(uint64_t pos, bool b = true) {
        uint64_t &w = m_words[pos >> 6];
        w = (w & ~(uint64_t(1) << (pos & 63))) | (uint64_t(b) << (pos & 63));
    }
    void set_bits(uint64_t pos, uint64_t value, uint64_t len) {
        if (!len) return;
        const uint64_t mask = len == 64 ? ~uint64_t(0) : (uint64_t(1) << len) - 1;
        const uint64_t w = pos >> 6, off = pos & 63;
        m_words[w] = (m_words[w] & ~(mask << off)) | (value << off);
        if (64 - off < len) m_words[w + 1] = (m_words[w + 1] & ~(mask >> (64 - off))) | (value >> (64 - off));
    }
    uint64_t size() const { return m_size; }
    std::vector<uint64_t> &words() { return m_words; }

  private:
    uint64_t m_size;
    std::vector<uint64_t> m_words;
};

class bit_vector {
  public:
    bit_vector() : m_size(0) {}
    explicit bit_vector(bit_vector_builder *b) : m_size(b->size()) { m_bits.swap(b->words()); }

    size_t size() const { return m_size; }
    uint64_t bytes() const { return sizeof(m_size) + bits::vec_bytes(m_bits); }
    const std::vector<uint64_t> &data() const { return m_bits; }
    uint64_t operator[](uint64_t i) const { return (m_bits[i >> 6] >> (i & 63)) & 1; }
    uint64_t get_bits(uint64_t pos, uint64_t len) const {
        if (!len) return 0;
        const uint64_t mask = len == 64 ? ~uint64_t(0) : (uint64_t(1) << len) - 1;
        const uint64_t w = pos >> 6, off = pos & 63;
        uint64_t v = m_bits[w] >> off;
        if (off + len > 64) v |= m_bits[w + 1] << (64 - off);
        return v & mask;
    }
    // Position of the next set bit at or after pos.
    uint64_t next_one(uint64_t pos) const {
        uint64_t w = pos >> 6;
        uint64_t word = m_bits[w] & (~uint64_t(0) << (pos & 63));
        while (!word) word = m_bits[++w];
        return (w << 6) + (uint64_t)__builtin_ctzll(word);
    }
    void swap(bit_vector &o) {
        std::swap(m_size, o.m_size);
        m_bits.swap(o.m_bits);
    }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_size);
        visitor.visit(m_bits);
    }

  private:
    size_t m_size;
    std::vector<uint64_t> m_bits;
};

// Fixed-width integer array: value i at bits [i*w, (i+1)*w), one spare word.
class compact_vector {
  public:
    class builder {
      public:
        builder() = default;
        builder(uint64_t n, uint64_t w) { resize(n, w); }
        void resize(uint64_t n, uint64_t w) {
            m_size = n;
            m_width = w;
            m_mask = w == 64 ? ~uint64_t(0) : (uint64_t(1) << w) - 1;
            m_pos = 0;
            m_bits.assign(bits::words_for(n * w) + 1, 0);
        }
        void push_back(uint64_t v) {
            if (!m_width) return;
            const uint64_t w = m_pos >> 6, off = m_pos & 63;
            m_bits[w] |= v << off;
            if (off + m_width > 64) m_bits[w + 1] |= v >> (64 - off);
            m_pos += m_width;
        }
        void build(compact_vector &cv) {
            cv.m_size = m_size;
            cv.m_width = m_width;
            cv.m_mask = m_mask;
            cv.m_bits.swap(m_bits);
            *this = builder();
        }

      private:
        uint64_t m_size = 0, m_width = 0, m_mask = 0, m_pos = 0;
        std::vector<uint64_t> m_bits;
    };

    compact_vector() : m_size(0), m_width(0), m_mask(0) {}

    template <typename Iterator>
    void build(Iterator begin, uint64_t n) {
        uint64_t mx = n ? *std::max_element(begin, begin + n) : 0;
        build(begin, n, bits::width_for(mx));
    }
    template <typename Iterator>
    void build(Iterator begin, uint64_t n, uint64_t w) {
        builder b(n, w);
        for (uint64_t i = 0; i < n; i++, ++begin) b.push_back(*begin);
        b.build(*this);
    }

    uint64_t access(uint64_t i) const {
        const uint64_t pos = i * m_width, w = pos >> 6, off = pos & 63;
        uint64_t v = m_bits[w] >> off;
        if (off + m_width > 64) v |= m_bits[w + 1] << (64 - off);
        return v & m_mask;
    }
    uint64_t size() const { return m_size; }
    uint64_t width() const { return m_width; }
    size_t bytes() const { return sizeof(m_size) + sizeof(m_width) + sizeof(m_mask) + bits::vec_bytes(m_bits); }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_size);
        visitor.visit(m_width);
        visitor.visit(m_mask);
        visitor.visit(m_bits);
    }

  private:
    uint64_t m_size, m_width, m_mask;
    std::vector<uint64_t> m_bits;
};

// Select index over the set bits of a bit_vector: one inventory entry per 4096
// set bits (its first position, or a pointer into the explicit positions when
// the block spans 2^16 bits or more), one 16-bit sub-entry per 64 set bits.
class darray1 {
  public:
    darray1() : m_positions(0) {}

    void build(const bit_vector &bv) {
        const std::vector<uint64_t> &data = bv.data();
        std::vector<uint64_t> cur;
        cur.reserve(kBlock);
        m_positions = 0;
        for (size_t wi = 0; wi < data.size(); wi++) {
            uint64_t word = data[wi];
            while (word) {
                const uint64_t pos = (wi << 6) + (uint64_t)__builtin_ctzll(word);
                word &= word - 1;
                if (pos >= bv.size()) break;
                cur.push_back(pos);
                if (cur.size() == kBlock) flush(cur);
                m_positions++;
            }
        }
        if (!cur.empty()) flush(cur);
    }

    uint64_t select(const bit_vector &bv, uint64_t idx) const {
        const int64_t block_pos = m_block_inventory[idx / kBlock];
        if (block_pos < 0) return m_overflow_positions[uint64_t(-block_pos - 1) + (idx % kBlock)];
        uint64_t pos = uint64_t(block_pos) + m_subblock_inventory[idx / kSub];
        uint64_t rem = idx % kSub;
        if (!rem) return pos;
        const std::vector<uint64_t> &data = bv.data();
        uint64_t wi = pos >> 6;
        uint64_t word = data[wi] & (~uint64_t(0) << (pos & 63));
        for (;;) {
            const uint64_t c = (uint64_t)__builtin_popcountll(word);
            if (rem < c) break;
            rem -= c;
            word = data[++wi];
        }
        return (wi << 6) + bits::select_in_word(word, rem);
    }

    uint64_t num_positions() const { return m_positions; }
    uint64_t bytes() const {
        return sizeof(m_positions) + bits::vec_bytes(m_block_inventory) + bits::vec_bytes(m_subblock_inventory) +
               bits::vec_bytes(m_overflow_positions);
    }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_positions);
        visitor.visit(m_block_inventory);
        visitor.visit(m_subblock_inventory);
        visitor.visit(m_overflow_positions);
    }

  private:
    static constexpr size_t kBlock = 4096, kSub = 64, kMaxSpan = 1 << 16;

    void flush(std::vector<uint64_t> &cur) {
        if (cur.back() - cur.front() < kMaxSpan) {
            m_block_inventory.push_back(int64_t(cur.front()));
            for (size_t i = 0; i < cur.size(); i += kSub) m_subblock_inventory.push_back(uint16_t(cur[i] - cur.front()));
        } else {
            m_block_inventory.push_back(-int64_t(m_overflow_positions.size()) - 1);
            m_overflow_positions.insert(m_overflow_positions.end(), cur.begin(), cur.end());
            for (size_t i = 0; i < cur.size(); i += kSub) m_subblock_inventory.push_back(uint16_t(-1));
        }
        cur.clear();
    }

    size_t m_positions;
    std::vector<int64_t> m_block_inventory;
    std::vector<uint16_t> m_subblock_inventory;
    std::vector<uint64_t> m_overflow_positions;
};

// Golomb-Rice codes: low l bits in a compact_vector, high part in unary.
class rice_sequence {
  public:
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) {
        if (n == 0) return;
        const uint64_t l = optimal_l(begin, n);
        bit_vector_builder high;
        compact_vector::builder low(n, l);
        const uint64_t low_mask = (uint64_t(1) << l) - 1;
        for (uint64_t i = 0; i < n; i++, ++begin) {
            const uint64_t v = *begin;
            low.push_back(v & low_mask);
            for (uint64_t u = v >> l; u; u--) high.push_back(false);
            high.push_back(true);
        }
        bit_vector(&high).swap(m_high_bits);
        low.build(m_low_bits);
        m_high_bits_d1.build(m_high_bits);
    }

    uint64_t access(uint64_t i) const {
        const int64_t start = i ? int64_t(m_high_bits_d1.select(m_high_bits, i - 1)) : -1;
        const int64_t end = int64_t(m_high_bits_d1.select(m_high_bits, i));
        return (uint64_t(end - start - 1) << m_low_bits.width()) | m_low_bits.access(i);
    }
    uint64_t size() const { return m_low_bits.size(); }
    uint64_t bytes() const { return m_high_bits.bytes() + m_high_bits_d1.bytes() + m_low_bits.bytes(); }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_high_bits);
        visitor.visit(m_high_bits_d1);
        visitor.visit(m_low_bits);
    }

  private:
    // Rice parameter for geometric values of mean sum/n (rice_sequence.hpp:15-21).
    template <typename Iterator>
    static uint64_t optimal_l(Iterator begin, uint64_t n) {
        const uint64_t sum = std::accumulate(begin, begin + n, uint64_t(0));
        const double p = n / (double(sum) + n);
        const double gold = std::log2(2.0 / (std::sqrt(5.0) + 1.0));
        const int64_t r = int64_t(std::ceil(std::log2(gold / std::log2(1.0 - p))));
        return uint64_t(std::max(int64_t(0), r));
    }

    bit_vector m_high_bits;
    darray1 m_high_bits_d1;
    compact_vector m_low_bits;
};

// Elias-Fano; with PrefixSum the input values are gaps and the sequence stores
// their prefix sums behind a leading zero.
template <bool PrefixSum = false>
class ef_sequence {
  public:
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n) {
        if (n == 0) return;
        uint64_t u = PrefixSum ? std::accumulate(begin, begin + n, uint64_t(0)) : *(begin + n - 1);
        const uint64_t stored = PrefixSum ? n + 1 : n;
        const uint64_t l = (u / stored) ? bits::msb(u / stored) : 0;
        bit_vector_builder high(stored + (u >> l) + 1);
        compact_vector::builder low(stored, l);
        const uint64_t low_mask = (uint64_t(1) << l) - 1;
        uint64_t last = 0;
        if (PrefixSum) {
            if (l) low.push_back(0);
            high.set(0, true);
        }
        for (uint64_t i = 0; i < n; i++, ++begin) {
            uint64_t v = *begin;
            if (PrefixSum) v += last;
            else if (i && v < last) throw std::runtime_error("ef_sequence is not sorted");
            if (l) low.push_back(v & low_mask);
            high.set((v >> l) + i + (PrefixSum ? 1 : 0), true);
            last = v;
        }
        bit_vector(&high).swap(m_high_bits);
        low.build(m_low_bits);
        m_high_bits_d1.build(m_high_bits);
    }

    uint64_t access(uint64_t i) const {
        return ((m_high_bits_d1.select(m_high_bits, i) - i) << m_low_bits.width()) | low(i);
    }
    uint64_t diff(uint64_t i) const {
        const uint64_t l = m_low_bits.width();
        const uint64_t pos = m_high_bits_d1.select(m_high_bits, i);
        const uint64_t h1 = pos - i;
        const uint64_t h2 = m_high_bits.next_one(pos + 1) - i - 1;
        return ((h2 << l) | low(i + 1)) - ((h1 << l) | low(i));
    }
    uint64_t size() const { return m_low_bits.size(); }
    uint64_t num_bits() const { return 8 * (m_high_bits.bytes() + m_high_bits_d1.bytes() + m_low_bits.bytes()); }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_high_bits);
        visitor.visit(m_high_bits_d1);
        visitor.visit(m_low_bits);
    }

  private:
    uint64_t low(uint64_t i) const { return m_low_bits.width() ? m_low_bits.access(i) : 0; }

    bit_vector m_high_bits;
    darray1 m_high_bits_d1;
    compact_vector m_low_bits;
};

// Simple dense coding: value v as the floor(log2(v+1)) low bits of v+1, with an
// Elias-Fano index of codeword start positions.
class sdc_sequence {
  public:
    sdc_sequence() : m_size(0) {}

    template <typename Iterator>
    void build(Iterator begin, uint64_t n) {
        m_size = n;
        uint64_t total = 0;
        Iterator it = begin;
        for (uint64_t i = 0; i < n; i++, ++it) total += bits::msb(uint64_t(*it) + 1);
        bit_vector_builder words(total);
        std::vector<uint64_t> starts;
        starts.reserve(n + 1);
        uint64_t pos = 0;
        for (uint64_t i = 0; i < n; i++, ++begin) {
            const uint64_t v = *begin;
            const uint64_t len = bits::msb(v + 1);
            if (len) words.set_bits(pos, v + 1 - (uint64_t(1) << len), len);
            starts.push_back(pos);
            pos += len;
        }
        starts.push_back(pos);
        bit_vector(&words).swap(m_codewords);
        m_index.encode(starts.data(), starts.size());
    }

    uint64_t access(uint64_t i) const {
        const uint64_t pos = m_index.access(i);
        const uint64_t len = m_index.access(i + 1) - pos;
        return m_codewords.get_bits(pos, len) + (uint64_t(1) << len) - 1;
    }
    uint64_t size() const { return m_size; }
    uint64_t bytes() const { return sizeof(m_size) + m_codewords.bytes() + m_index.num_bits() / 8; }

    template <typename Visitor>
    void visit(Visitor &visitor) {
        visitor.visit(m_size);
        visitor.visit(m_codewords);
        visitor.visit(m_index);
    }

  private:
    uint64_t m_size;
    bit_vector m_codewords;
    ef_sequence<false> m_index;
};

}  // namespace phobicgpu
