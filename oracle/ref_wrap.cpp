// Oracle (test infrastructure only): C entry points over the reference's own
// host headers, compiled in place from the reference checkout by
// oracle/Makefile into oracle/_ref/libphobic_ref.so.
//
// What runs here is the reference's code, unmodified:
//   - xxhash::hash for u64, std::string, pair<u64,u64> and Key (hasher.hpp:30-67)
//   - MPHFconfig / bucketers fulcrum construction (mphf_config.h:26-64)
//   - MPHF::setData encoders and MPHF::operator() query (mphf.hpp:65-86)
// The shaders (GLSL) cannot run here; their restatement lives in orc_build.c.
#include <numeric>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "phobicGpu/mphf.hpp"
#include "encoders/pilotEncoders/mono_encoders.hpp"
#include "encoders/partitionOffsetEnocders/diff_partition_offset_encoder.hpp"
#include "encoders/partitionOffsetEnocders/direct_partition_offset_encoder.hpp"

using namespace phobicgpu;

namespace {

// Serialises an encoder through its visit() methods: scalars as raw bytes,
// vectors as a size_t count followed by their elements.
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

// MPHF exposes no visit(): the pilot encoder is reached through the public
// getPilotEncoder(), the offsets encoder is rebuilt from the same offsets
// (identical input, identical bytes).
template <typename PilotEnc, typename OffEnc>
size_t encode_impl(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, double lambda, uint32_t P,
                   uint8_t *out, size_t cap, double *bits_per_key, float tradeoff) {
    MPHFconfig config(lambda, P);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * config.bucketCountPerPartition);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<PilotEnc, OffEnc, xxhash> f;
    if constexpr (std::is_same_v<PilotEnc, interleaved_encoder_dual<rice, compact>>) {
        f.getPilotEncoder().setEncoderTradeoff(tradeoff);
    }
    f.setData(pil, offs, partitions, config);
    OffEnc off;
    off.encode(offs.begin(), config.partitionSize, partitions + 1);
    ByteSaver s;
    f.getPilotEncoder().visit(s);
    off.visit(s);
    if (bits_per_key) *bits_per_key = f.getBitsPerKey();
    if (out && s.out.size() <= cap) std::memcpy(out, s.out.data(), s.out.size());
    return s.out.size();
}

template <typename OffEnc>
size_t encode_pilot_kind(int pilot_kind, const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions,
                         double lambda, uint32_t P, uint8_t *out, size_t cap, double *bpk, float tradeoff) {
    switch (pilot_kind) {
    case 0: return encode_impl<interleaved_encoder<compact>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 1: return encode_impl<interleaved_encoder<dictionary>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 2: return encode_impl<interleaved_encoder<rice>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 3: return encode_impl<mono_encoder<compact>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 4: return encode_impl<mono_encoder<dictionary>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 5: return encode_impl<interleaved_encoder_dual<rice, compact>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 6: return encode_impl<interleaved_encoder<elias_fano>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 7: return encode_impl<interleaved_encoder<sdc>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    case 8: return encode_impl<mono_encoder<rice>, OffEnc>(pilots, offsets, partitions, lambda, P, out, cap, bpk, tradeoff);
    default: return 0;
    }
}

void key_out(const Key &k, uint32_t *o) {
    o[0] = k.partitioner;
    o[1] = k.bucketer;
    o[2] = k.lower1;
    o[3] = k.lower2;
}

}  // namespace

extern "C" {

// xxhash::hash over four key types (hasher.hpp:30-67).
void ref_hash_u64(const uint64_t *keys, uint64_t n, uint32_t *keys4) {
    for (uint64_t i = 0; i < n; i++) key_out(xxhash::hash(keys[i]), keys4 + 4 * i);
}
void ref_hash_pairs(const uint64_t *pairs, uint64_t n, uint32_t *keys4) {
    for (uint64_t i = 0; i < n; i++)
        key_out(xxhash::hash(std::pair<uint64_t, uint64_t>(pairs[2 * i], pairs[2 * i + 1])), keys4 + 4 * i);
}
void ref_hash_keys16(const uint32_t *in4, uint64_t n, uint32_t *keys4) {
    for (uint64_t i = 0; i < n; i++)
        key_out(xxhash::hash(Key(in4[4 * i], in4[4 * i + 1], in4[4 * i + 2], in4[4 * i + 3])), keys4 + 4 * i);
}
void ref_hash_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint32_t *keys4) {
    for (uint64_t i = 0; i < n; i++) {
        std::string s(reinterpret_cast<const char *>(bytes + offsets[i]), offsets[i + 1] - offsets[i]);
        key_out(xxhash::hash(s), keys4 + 4 * i);
    }
}

// MPHFconfig(λ, P) or MPHFconfig(Bucketer*, λ, P); bucketer 0 = Opt, 1 = Uniform, 2 = Skew.
uint32_t ref_config(double lambda, uint32_t P, int bucketer, int bucketer_ctor, uint32_t *fulcs,
                    uint32_t *partition_max_size) {
    Bucketer *b = nullptr;
    if (bucketer == 1) b = new UniformBucketer();
    else if (bucketer == 2) b = new SkewBucketer();
    else b = new OptBucketer();
    MPHFconfig cfg = bucketer_ctor ? MPHFconfig(b, lambda, P) : MPHFconfig(lambda, P);
    delete b;
    const std::vector<uint32_t> &f = cfg.getFulcs();
    std::memcpy(fulcs, f.data(), f.size() * sizeof(uint32_t));
    if (partition_max_size) *partition_max_size = cfg.partitionMaxSize();
    return cfg.bucketCountPerPartition;
}

// MPHF::setData (mphf.hpp:65-75) followed by a visit() serialisation of the
// pilot encoder and the partition-offset encoder.  offset_kind 0 = diff, 1 = direct
// (both over compact).  Returns the byte count (writes only if it fits in cap).
size_t ref_encode(int pilot_kind, int offset_kind, const uint32_t *pilots, const uint32_t *offsets,
                  uint32_t partitions, double lambda, uint32_t P, float tradeoff, uint8_t *out, size_t cap,
                  double *bits_per_key) {
    if (offset_kind == 1)
        return encode_pilot_kind<direct_partition_encoder<compact>>(pilot_kind, pilots, offsets, partitions, lambda, P,
                                                                    out, cap, bits_per_key, tradeoff);
    return encode_pilot_kind<diff_partition_encoder<compact>>(pilot_kind, pilots, offsets, partitions, lambda, P, out,
                                                              cap, bits_per_key, tradeoff);
}

// MPHF::operator() (mphf.hpp:77-86) for u64 keys, with interleaved compact pilots.
void ref_query_u64(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, double lambda, uint32_t P,
                   const uint64_t *keys, uint64_t n, uint32_t *out) {
    MPHFconfig config(lambda, P);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * config.bucketCountPerPartition);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<interleaved_encoder<compact>, diff_partition_encoder<compact>, xxhash> f;
    f.setData(pil, offs, partitions, config);
    for (uint64_t i = 0; i < n; i++) out[i] = f(keys[i]);
}

}  // extern "C"
