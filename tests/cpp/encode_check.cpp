// Test harness: the C++ layer's encoders behind a C entry point with the same
// arguments as the reference wrapper's ref_encode (oracle/ref_wrap.cpp), so the
// tests can compare serialised bytes of the two implementations.
#include <cstring>
#include <type_traits>
#include <vector>

#include "phobic_gpu_mphf.hpp"

using namespace phobicgpu;

namespace {

template <typename PilotEnc, typename OffEnc>
size_t encode_impl(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, double lambda, uint32_t P,
                   uint8_t *out, size_t cap, double *bpk, float tradeoff) {
    MPHFconfig config(lambda, P);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * config.bucketCountPerPartition);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<PilotEnc, OffEnc, xxhash> f;
    if constexpr (std::is_same_v<PilotEnc, interleaved_encoder_dual<rice, compact>>) f.getPilotEncoder().setEncoderTradeoff(tradeoff);
    f.setData(pil, offs, partitions, config);
    ByteSaver s;
    f.getPilotEncoder().visit(s);
    f.getPartitionOffsetEncoder().visit(s);
    if (bpk) *bpk = f.getBitsPerKey();
    if (out && s.out.size() <= cap) std::memcpy(out, s.out.data(), s.out.size());
    return s.out.size();
}

template <typename OffEnc>
size_t by_kind(int kind, const uint32_t *p, const uint32_t *o, uint32_t parts, double l, uint32_t P, uint8_t *out,
               size_t cap, double *bpk, float t) {
    switch (kind) {
    case 0: return encode_impl<interleaved_encoder<compact>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 1: return encode_impl<interleaved_encoder<dictionary>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 2: return encode_impl<interleaved_encoder<rice>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 3: return encode_impl<mono_encoder<compact>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 4: return encode_impl<mono_encoder<dictionary>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 5: return encode_impl<interleaved_encoder_dual<rice, compact>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 6: return encode_impl<interleaved_encoder<elias_fano>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 7: return encode_impl<interleaved_encoder<sdc>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    case 8: return encode_impl<mono_encoder<rice>, OffEnc>(p, o, parts, l, P, out, cap, bpk, t);
    default: return 0;
    }
}

// Query every key through the encoded function (checks access paths of all encoders).
template <typename PilotEnc>
int query_impl(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, double lambda, uint32_t P,
               const uint64_t *keys, uint64_t n, uint32_t *out) {
    MPHFconfig config(lambda, P);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * config.bucketCountPerPartition);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<PilotEnc, diff_partition_encoder<compact>, xxhash> f;
    f.setData(pil, offs, partitions, config);
    for (uint64_t i = 0; i < n; i++) out[i] = f(keys[i]);
    return 0;
}

// Encode with setData, serialise, load the bytes into a fresh MPHF with
// loadEncoded and query every key through both: 0 when every slot agrees and the
// reloaded function re-serialises to the same bytes, 1 on a difference, 2 when
// loadEncoded rejects the bytes, 3 when it accepts them with one byte missing.
template <typename PilotEnc, typename OffEnc>
int roundtrip_impl(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, double lambda, uint32_t P,
                   const uint64_t *keys, uint64_t n) {
    MPHFconfig config(lambda, P);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * config.bucketCountPerPartition);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<PilotEnc, OffEnc, xxhash> f, g, h;
    f.setData(pil, offs, partitions, config);
    ByteSaver s;
    f.getPilotEncoder().visit(s);
    f.getPartitionOffsetEncoder().visit(s);
    if (!g.loadEncoded(s.out.data(), s.out.size(), partitions, config)) return 2;
    if (!s.out.empty() && h.loadEncoded(s.out.data(), s.out.size() - 1, partitions, config)) return 3;
    for (uint64_t i = 0; i < n; i++)
        if (f(keys[i]) != g(keys[i])) return 1;
    ByteSaver t;
    g.getPilotEncoder().visit(t);
    g.getPartitionOffsetEncoder().visit(t);
    return t.out == s.out ? 0 : 1;
}

}  // namespace

extern "C" int mine_roundtrip(int pilot_kind, int offset_kind, const uint32_t *pilots, const uint32_t *offsets,
                              uint32_t partitions, double lambda, uint32_t P, const uint64_t *keys, uint64_t n) {
    const bool direct = offset_kind == 1;
    if (pilot_kind == 0)
        return direct ? roundtrip_impl<interleaved_encoder<compact>, direct_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n)
                      : roundtrip_impl<interleaved_encoder<compact>, diff_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n);
    if (pilot_kind == 3)
        return direct ? roundtrip_impl<mono_encoder<compact>, direct_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n)
                      : roundtrip_impl<mono_encoder<compact>, diff_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n);
    if (pilot_kind == 1)
        return direct ? roundtrip_impl<interleaved_encoder<dictionary>, direct_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n)
                      : roundtrip_impl<interleaved_encoder<dictionary>, diff_partition_encoder<compact>>(
                            pilots, offsets, partitions, lambda, P, keys, n);
    return -1;
}

// A pilot-layout file (written by the Python binding) loaded with loadPilotLayout,
// encoded with setData (interleaved compact + diff compact), saved with
// MPHF::save, loaded again with MPHF::load, and every key queried through both:
// 0 when all agree, 1 on a difference, 2 when the layout file is rejected, 3 when
// MPHF::load rejects the saved bytes, 4 when it accepts them truncated.
extern "C" int mine_layout_and_save(const char *path, double lambda, const uint64_t *keys, uint64_t n) {
    PilotLayout l;
    if (!loadPilotLayout(path, &l)) return 2;
    MPHFconfig config(lambda, l.partition_size);
    FastQueryMphf f, g, h;
    f.setData(l.pilots, l.offsets, l.partitions, config);
    std::vector<uint8_t> bytes = f.save();
    if (!g.load(bytes.data(), bytes.size(), l.partition_size)) return 3;
    if (!bytes.empty() && h.load(bytes.data(), bytes.size() - 1, l.partition_size)) return 4;
    for (uint64_t i = 0; i < n; i++)
        if (f(keys[i]) != g(keys[i])) return 1;
    return g.save() == bytes ? 0 : 1;
}

extern "C" size_t mine_encode(int pilot_kind, int offset_kind, const uint32_t *pilots, const uint32_t *offsets,
                              uint32_t partitions, double lambda, uint32_t P, float tradeoff, uint8_t *out, size_t cap,
                              double *bits_per_key) {
    if (offset_kind == 1)
        return by_kind<direct_partition_encoder<compact>>(pilot_kind, pilots, offsets, partitions, lambda, P, out, cap,
                                                          bits_per_key, tradeoff);
    return by_kind<diff_partition_encoder<compact>>(pilot_kind, pilots, offsets, partitions, lambda, P, out, cap,
                                                    bits_per_key, tradeoff);
}

extern "C" int mine_query(int pilot_kind, const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions,
                          double lambda, uint32_t P, const uint64_t *keys, uint64_t n, uint32_t *out) {
    switch (pilot_kind) {
    case 0: return query_impl<interleaved_encoder<compact>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 1: return query_impl<interleaved_encoder<dictionary>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 2: return query_impl<interleaved_encoder<rice>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 3: return query_impl<mono_encoder<compact>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 5: return query_impl<interleaved_encoder_dual<rice, compact>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 6: return query_impl<interleaved_encoder<elias_fano>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 7: return query_impl<interleaved_encoder<sdc>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    case 8: return query_impl<mono_encoder<rice>>(pilots, offsets, partitions, lambda, P, keys, n, out);
    default: return -1;
    }
}
