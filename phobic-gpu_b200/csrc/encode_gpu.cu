// Encoding of a build's result on the device, for the encoders made of compact
// vectors: interleaved_encoder<compact> and mono_encoder<compact> pilots
// (include/encoders/pilotEncoders/interleaved_encoder.hpp:8-15, mono_encoders.hpp),
// diff_partition_encoder<compact> and direct_partition_encoder<compact> offsets
// (include/encoders/partitionOffsetEnocders/*.hpp, base/linear_diff_encoder.hpp:15-28).
// This is Mphf::setData (include/phobicGpu/mphf.hpp:65-75) without the host pass
// over the pilots.
//
// Every compact vector is written as the host encoders serialise it, in visit
// order: size, width, mask (u64 each), then its words as a vector (u64 count,
// count = ceil(size * width / 64) + 1, then the words).  Value i occupies bits
// [i w, i w + w) of the little-endian word array; width = bit length of the
// largest value, at least 1 (compact_vector.hpp build).  The bytes equal
// phobic_encode's for the same arrays.
//
//   k_colmax     per column (an interleaved column of `partitions` pilots, or the
//                one mono column of all pilots): largest value
//   k_codemax    largest partition-offset code (zig-zag difference to i * P, or
//                the offset itself)
//   k_pack       one thread per output word of every column; writes the headers
//
// A column's words depend only on its values and width, so all columns are
// written by one launch from a table of (values, count, width, byte offset).
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "kernels.cuh"

namespace phobicb200 {

namespace {

constexpr int kEncThreads = 256;

// One compact vector of the output.
struct EncColumn {
    const uint32_t *vals;  // pilot column (null: the partition-offset codes)
    uint64_t n;            // values
    uint64_t out;          // byte offset of its header in the output
    uint32_t width;
    uint32_t pad;
};

// Code of partition offset i (linear_diff_encoder.hpp:15-28 for diff, the value itself for direct).
__device__ __forceinline__ uint64_t offset_code(const uint32_t *off, uint64_t i, uint32_t psize, bool diff) {
    const uint64_t v = off[i];
    if (!diff) return v;
    const int64_t d = (int64_t)v - (int64_t)(i * psize);
    const uint64_t a = (uint64_t)(d < 0 ? -d : d);
    return (a << 1) | (uint64_t)(d > 0);
}

__device__ __forceinline__ uint64_t words_for(uint64_t bits) { return (bits + 63) / 64; }

// Largest value of column blockIdx.y, per CTA chunk, into maxes[y] (atomicMax).
__global__ void __launch_bounds__(kEncThreads) k_colmax(const uint32_t *pilots, uint64_t per_col, uint32_t *maxes) {
    const uint32_t *v = pilots + (uint64_t)blockIdx.y * per_col;
    uint32_t m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < per_col; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, __ldg(v + i));
    m = __reduce_max_sync(kFullMask, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(&maxes[blockIdx.y], m);
}

__global__ void __launch_bounds__(kEncThreads) k_codemax(const uint32_t *off, uint64_t count, uint32_t psize, int diff,
                                                         unsigned long long *mx) {
    unsigned long long m = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, (unsigned long long)offset_code(off, i, psize, diff != 0));
    for (int d = 16; d; d >>= 1) m = max(m, __shfl_xor_sync(kFullMask, m, d));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(mx, m);
}

// Word t of column blockIdx.x / per_col (t = index among the vector's words, the
// column's CTAs striding over them; the header's four u64 are written by t = 0).
// Words past ceil(n w / 64) are zero.
__global__ void __launch_bounds__(kEncThreads) k_pack(const EncColumn *cols, uint32_t per_col, const uint32_t *off,
                                                      uint32_t psize, int diff, uint8_t *out) {
    const EncColumn c = cols[blockIdx.x / per_col];
    const uint64_t chunk = blockIdx.x % per_col;
    const uint64_t w = c.width;
    const uint64_t words = words_for(c.n * w) + 1;
    uint64_t *hdr = reinterpret_cast<uint64_t *>(out + c.out);
    uint64_t *bits = hdr + 4;
    for (uint64_t t = chunk * blockDim.x + threadIdx.x; t < words; t += (uint64_t)per_col * blockDim.x) {
        if (t == 0) {
            hdr[0] = c.n;
            hdr[1] = w;
            hdr[2] = w == 64 ? ~0ull : (1ull << w) - 1;
            hdr[3] = words;
        }
        const uint64_t lo = 64 * t, hi = lo + 64;  // bits of this word
        uint64_t word = 0;
        if (lo < c.n * w) {
            const uint64_t i0 = lo / w;
            uint64_t i1 = (hi - 1) / w;
            if (i1 >= c.n) i1 = c.n - 1;
            for (uint64_t i = i0; i <= i1; i++) {
                const uint64_t v = c.vals ? (uint64_t)__ldg(c.vals + i) : offset_code(off, i, psize, diff != 0);
                const uint64_t pos = i * w;
                word |= pos >= lo ? v << (pos - lo) : v >> (lo - pos);
            }
        }
        bits[t] = word;
    }
}

uint32_t width_of(uint64_t max_value) { return max_value ? 64 - __builtin_clzll(max_value) : 1; }
uint64_t host_words(uint64_t bits) { return (bits + 63) / 64; }
uint64_t vector_bytes(uint64_t n, uint32_t w) { return 32 + 8 * (host_words(n * w) + 1); }

}  // namespace

phobic_status run_encode_gpu(Worker &w, DeviceArena &out_arena, int pilot_encoder, int offset_encoder,
                             const phobic_result *built, uint32_t partitions, const phobic_params *params,
                             uint8_t *out, size_t cap, int out_on_device, size_t *size, double *bits_per_key,
                             std::string *err) {
    if (!built || !params || !size || (pilot_encoder != 0 && pilot_encoder != 3) ||
        (offset_encoder != 0 && offset_encoder != 1) || params->buckets == 0 || params->partition_size == 0) {
        if (err) *err = "phobic_encode_gpu: unsupported encoder or missing argument";
        return PHOBIC_ERR_INVALID;
    }
    const uint64_t B = params->buckets, P = partitions;
    const uint64_t npil = B * P, noff = P + 1;
    const bool mono = pilot_encoder == 3;
    const uint32_t cols = mono ? 1u : (uint32_t)B;
    PHB_TRY(cudaSetDevice(w.device), "cudaSetDevice");
    PHB_TRY(w.pinned.reserve(4096 + 4 * (size_t)cols + sizeof(EncColumn) * (cols + 1)), "pinned");
    cudaStream_t s = w.stream;

    // Inputs on the device, the maxima, the column table.
    const size_t need = align256(4 * npil) + align256(4 * noff) + align256(4 * (size_t)cols) + align256(8) +
                        align256(sizeof(EncColumn) * (cols + 1)) + 4096;
    w.arena.reset();
    PHB_TRY(w.arena.reserve(need), "device arena");
    const uint32_t *d_pil = built->pilots, *d_off = built->partition_offsets;
    if (!built->on_device) {
        uint32_t *a = static_cast<uint32_t *>(w.arena.take(4 * npil));
        uint32_t *b = static_cast<uint32_t *>(w.arena.take(4 * noff));
        if (npil) PHB_TRY(cudaMemcpyAsync(a, built->pilots, 4 * npil, cudaMemcpyHostToDevice, s), "H2D pilots");
        PHB_TRY(cudaMemcpyAsync(b, built->partition_offsets, 4 * noff, cudaMemcpyHostToDevice, s), "H2D offsets");
        d_pil = a, d_off = b;
    }
    uint32_t *d_max = static_cast<uint32_t *>(w.arena.take(4 * (size_t)cols));
    unsigned long long *d_cmax = static_cast<unsigned long long *>(w.arena.take(8));
    EncColumn *d_cols = static_cast<EncColumn *>(w.arena.take(sizeof(EncColumn) * (cols + 1)));
    PHB_TRY(cudaMemsetAsync(d_max, 0, 4 * (size_t)cols, s), "memset");
    PHB_TRY(cudaMemsetAsync(d_cmax, 0, 8, s), "memset");
    const uint64_t per_col = mono ? npil : P;
    if (per_col) {
        const uint32_t gx = (uint32_t)std::min<uint64_t>((per_col + kEncThreads * 8 - 1) / (kEncThreads * 8),
                                                         mono ? (uint64_t)w.sm_count * 8 : 64);
        k_colmax<<<dim3(gx, cols), kEncThreads, 0, s>>>(d_pil, per_col, d_max);
        PHB_TRY(cudaGetLastError(), "k_colmax");
    }
    const uint32_t psize = params->partition_size;
    const int diff = offset_encoder == 0;
    k_codemax<<<(uint32_t)std::min<uint64_t>((noff + kEncThreads - 1) / kEncThreads, 1024), kEncThreads, 0, s>>>(
        d_off, noff, psize, diff, d_cmax);
    PHB_TRY(cudaGetLastError(), "k_codemax");
    uint8_t *hp = static_cast<uint8_t *>(w.pinned.data());
    uint32_t *h_max = reinterpret_cast<uint32_t *>(hp + 64);
    unsigned long long *h_cmax = reinterpret_cast<unsigned long long *>(hp);
    uint32_t *h_n = reinterpret_cast<uint32_t *>(hp + 8);
    PHB_TRY(cudaMemcpyAsync(h_max, d_max, 4 * (size_t)cols, cudaMemcpyDeviceToHost, s), "D2H maxima");
    PHB_TRY(cudaMemcpyAsync(h_cmax, d_cmax, 8, cudaMemcpyDeviceToHost, s), "D2H maxima");
    PHB_TRY(cudaMemcpyAsync(h_n, d_off + P, 4, cudaMemcpyDeviceToHost, s), "D2H n");
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    phobic_status st = wait_event(w.ev[7], w.timeout_ms, err);
    if (st != PHOBIC_OK) return st;

    // Column table and sizes (host), in visit order: pilot columns, then the offsets.
    EncColumn *h_cols = reinterpret_cast<EncColumn *>(hp + 64 + align256(4 * (size_t)cols));
    uint64_t total = 0;
    for (uint32_t j = 0; j < cols; j++) {
        const uint32_t wd = width_of(h_max[j]);
        h_cols[j] = EncColumn{d_pil + (uint64_t)j * per_col, per_col, total, wd, 0};
        total += vector_bytes(per_col, wd);
    }
    const uint32_t wo = width_of(*h_cmax);
    h_cols[cols] = EncColumn{nullptr, noff, total, wo, 0};
    total += vector_bytes(noff, wo);
    *size = total;
    if (bits_per_key) {
        // getBitsPerKey (mphf.hpp:88-91): encoder bits (8 per serialised byte), fulcrums and partition count.
        const uint64_t n = *h_n;
        *bits_per_key = n ? (double)(float(total * 8 + 32 * (uint64_t)kFulcrums + 32 * P) / float(n)) : 0.0;
    }
    if (!out) return PHOBIC_OK;

    // The kernel stores 8-byte words: a device destination that is too small or not
    // 8-byte aligned is written through the staging buffer.
    uint8_t *d_out = out;
    if (!out_on_device || cap < total || (reinterpret_cast<uintptr_t>(out) & 7)) {
        PHB_TRY(out_arena.reserve(total), "device output");
        out_arena.reset();
        d_out = static_cast<uint8_t *>(out_arena.take(total));
    }
    PHB_TRY(cudaMemcpyAsync(d_cols, h_cols, sizeof(EncColumn) * (cols + 1), cudaMemcpyHostToDevice, s), "H2D table");
    uint64_t max_words = 0;
    for (uint32_t j = 0; j <= cols; j++) max_words = std::max(max_words, host_words(h_cols[j].n * h_cols[j].width) + 1);
    const uint64_t per = std::min<uint64_t>((max_words + kEncThreads - 1) / kEncThreads,
                                            std::max<uint64_t>(1, (uint64_t)w.sm_count * 16 / (cols + 1)));
    k_pack<<<(uint32_t)(per * (cols + 1)), kEncThreads, 0, s>>>(d_cols, (uint32_t)per, d_off, psize, diff, d_out);
    PHB_TRY(cudaGetLastError(), "k_pack");
    if (d_out != out) {
        const size_t ncopy = std::min<size_t>(cap, total);
        if (ncopy)
            PHB_TRY(cudaMemcpyAsync(out, d_out, ncopy, out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    s),
                    "copy out");
    }
    PHB_TRY(cudaEventRecord(w.ev[7], s), "event");
    return wait_event(w.ev[7], w.timeout_ms, err);
}

}  // namespace phobicb200
