// phobic_encode: the host encoding step (Mphf::setData, include/phobicGpu/mphf.hpp:65-75)
// behind the C ABI, using the C++ layer's encoders (phobic-gpu_b200/cpp).
#include <cstring>
#include <type_traits>
#include <vector>

#include "phobic_b200.h"
#include "phobic_gpu_mphf.hpp"

using namespace phobicgpu;

namespace {

// An MPHFconfig with the caller's table (the encoders read partitionSize and B).
MPHFconfig config_from(const phobic_params *p) {
    MPHFconfig c(double(p->partition_size) / double(p->buckets), p->partition_size);
    c.bucketCountPerPartition = p->buckets;
    return c;
}

template <typename PilotEnc, typename OffEnc>
size_t encode_as(const uint32_t *pilots, const uint32_t *offsets, uint32_t partitions, const phobic_params *p,
                 float tradeoff, uint8_t *out, size_t cap, double *bpk) {
    MPHFconfig config = config_from(p);
    std::vector<uint32_t> pil(pilots, pilots + (size_t)partitions * p->buckets);
    std::vector<uint32_t> offs(offsets, offsets + partitions + 1);
    MPHF<PilotEnc, OffEnc, xxhash> f;
    if constexpr (std::is_same_v<PilotEnc, interleaved_encoder_dual<rice, compact>>) f.getPilotEncoder().setEncoderTradeoff(tradeoff);
    f.setData(pil, offs, partitions, config);
    ByteSaver s;
    f.getPilotEncoder().visit(s);
    f.getPartitionOffsetEncoder().visit(s);
    if (bpk) *bpk = partitions ? f.getBitsPerKey() : 0.0;
    if (out) std::memcpy(out, s.out.data(), std::min(cap, s.out.size()));
    return s.out.size();
}

template <typename OffEnc>
size_t by_pilot(int kind, const uint32_t *p, const uint32_t *o, uint32_t parts, const phobic_params *pp, float t,
                uint8_t *out, size_t cap, double *bpk) {
    switch (kind) {
    case 0: return encode_as<interleaved_encoder<compact>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 1: return encode_as<interleaved_encoder<dictionary>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 2: return encode_as<interleaved_encoder<rice>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 3: return encode_as<mono_encoder<compact>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 4: return encode_as<mono_encoder<dictionary>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 5: return encode_as<interleaved_encoder_dual<rice, compact>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 6: return encode_as<interleaved_encoder<elias_fano>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    case 7: return encode_as<interleaved_encoder<sdc>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    default: return encode_as<mono_encoder<rice>, OffEnc>(p, o, parts, pp, t, out, cap, bpk);
    }
}

}  // namespace

extern "C" phobic_status phobic_encode(int pilot_encoder, int offset_encoder, const uint32_t *pilots,
                                       const uint32_t *partition_offsets, uint32_t partitions,
                                       const phobic_params *params, float tradeoff, uint8_t *out, size_t cap,
                                       size_t *size, double *bits_per_key) {
    if (!params || !size || !partition_offsets || (partitions && !pilots) || pilot_encoder < 0 || pilot_encoder > 8 ||
        offset_encoder < 0 || offset_encoder > 1 || params->buckets == 0 || params->partition_size == 0)
        return PHOBIC_ERR_INVALID;
    *size = offset_encoder == 1
                ? by_pilot<direct_partition_encoder<compact>>(pilot_encoder, pilots, partition_offsets, partitions, params,
                                                              tradeoff, out, cap, bits_per_key)
                : by_pilot<diff_partition_encoder<compact>>(pilot_encoder, pilots, partition_offsets, partitions, params,
                                                            tradeoff, out, cap, bits_per_key);
    return PHOBIC_OK;
}
