// Key hashing and key mapping shared by the host library and the sm_100a kernels.
//
// * XXH3-128 with seed 0 (the reference's initial hash, include/phobicGpu/
//   hasher.hpp:30-67, which calls XXH128 from the xxHash library).  Written
//   from the published XXH3 specification; stable output since xxHash 0.8.0.
// * Key split {partitioner, bucketer, lower1, lower2} = 32-bit words of
//   (low64, high64) in little-endian order (hasher.hpp:7-20, :42-48).
// * Partition and bucket mapping (shaders/key_mapping.glsl:9-49; the 64-bit
//   query form in include/phobicGpu/mphf.hpp:42-49).
// * Pilot hash (shaders/hashing.glsl:11-17, mphf.hpp:23-40).
//
// Compiles as plain C++17 (user code, host library) and as CUDA (kernels).
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define PHB_HD __host__ __device__ __forceinline__
#else
#define PHB_HD inline
#endif

namespace phobicb200 {

constexpr uint32_t kFulcrums = 2048;  // shaders/constants.glsl:1
constexpr uint32_t kBins = 256;       // MPHFconfig::sortingBins, mphf_config.h:28

struct Key4 {
    uint32_t partitioner;
    uint32_t bucketer;
    uint32_t lower1;
    uint32_t lower2;
};

namespace xxh3 {

constexpr uint64_t kP32_1 = 0x9E3779B1ULL;
constexpr uint64_t kP32_2 = 0x85EBCA77ULL;
constexpr uint64_t kP32_3 = 0xC2B2AE3DULL;
constexpr uint64_t kP64_1 = 0x9E3779B185EBCA87ULL;
constexpr uint64_t kP64_2 = 0xC2B2AE3D27D4EB4FULL;
constexpr uint64_t kP64_3 = 0x165667B19E3779F9ULL;
constexpr uint64_t kP64_4 = 0x85EBCA77C2B2AE63ULL;
constexpr uint64_t kP64_5 = 0x27D4EB2F165667C5ULL;
constexpr uint64_t kMx1 = 0x165667919E3779F9ULL;
constexpr uint64_t kMx2 = 0x9FB21C651E98DF25ULL;

// The default secret as 24 little-endian 64-bit words (xxHash specification).
// Word w holds secret bytes [8w, 8w+8); unaligned reads combine two words.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint64_t secret_word(unsigned w) {
    // Written as a switch so that the device side needs no memory table and
    // constant-folds every fixed-offset read.
    switch (w) {
    case 0: return 0xbe4ba423396cfeb8ULL;
    case 1: return 0x1cad21f72c81017cULL;
    case 2: return 0xdb979083e96dd4deULL;
    case 3: return 0x1f67b3b7a4a44072ULL;
    case 4: return 0x78e5c0cc4ee679cbULL;
    case 5: return 0x2172ffcc7dd05a82ULL;
    case 6: return 0x8e2443f7744608b8ULL;
    case 7: return 0x4c263a81e69035e0ULL;
    case 8: return 0xcb00c391bb52283cULL;
    case 9: return 0xa32e531b8b65d088ULL;
    case 10: return 0x4ef90da297486471ULL;
    case 11: return 0xd8acdea946ef1938ULL;
    case 12: return 0x3f349ce33f76faa8ULL;
    case 13: return 0x1d4f0bc7c7bbdcf9ULL;
    case 14: return 0x3159b4cd4be0518aULL;
    case 15: return 0x647378d9c97e9fc8ULL;
    case 16: return 0xc3ebd33483acc5eaULL;
    case 17: return 0xeb6313faffa081c5ULL;
    case 18: return 0x49daf0b751dd0d17ULL;
    case 19: return 0x9e68d429265516d3ULL;
    case 20: return 0xfca1477d58be162bULL;
    case 21: return 0xce31d07ad1b8f88fULL;
    case 22: return 0x280416958f3acb45ULL;
    case 23: return 0x7e404bbbcafbd7afULL;
    default: return 0;
    }
}

// Secret bytes [off, off+8) as a little-endian word, any byte offset < 185.
PHB_HD uint64_t sec64(unsigned off) {
    unsigned w = off >> 3, sh = (off & 7) * 8;
    uint64_t lo = secret_word(w);
    return sh ? (lo >> sh) | (secret_word(w + 1) << (64 - sh)) : lo;
}
PHB_HD uint32_t sec32(unsigned off) { return (uint32_t)sec64(off); }

PHB_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}
PHB_HD uint64_t fold64(uint64_t a, uint64_t b) { return (a * b) ^ mulhi64(a, b); }
PHB_HD uint64_t bswap64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return ((uint64_t)__byte_perm((uint32_t)x, 0, 0x0123) << 32) | __byte_perm((uint32_t)(x >> 32), 0, 0x0123);
#else
    return __builtin_bswap64(x);
#endif
}
PHB_HD uint32_t bswap32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __byte_perm(x, 0, 0x0123);
#else
    return __builtin_bswap32(x);
#endif
}
PHB_HD uint64_t avalanche3(uint64_t h) {
    h ^= h >> 37;
    h *= kMx1;
    return h ^ (h >> 32);
}
PHB_HD uint64_t avalanche64(uint64_t h) {
    h ^= h >> 33;
    h *= kP64_2;
    h ^= h >> 29;
    h *= kP64_3;
    return h ^ (h >> 32);
}

struct H128 {
    uint64_t lo, hi;
};

// 4..8 byte inputs given as lo32 = first four bytes, hi32 = last four bytes.
PHB_HD H128 len4to8(uint32_t first4, uint32_t last4, uint32_t len) {
    uint64_t keyed = ((uint64_t)first4 | ((uint64_t)last4 << 32)) ^ (sec64(16) ^ sec64(24));
    uint64_t m = kP64_1 + ((uint64_t)len << 2);
    uint64_t lo = keyed * m;
    uint64_t hi = mulhi64(keyed, m);
    hi += lo << 1;
    lo ^= hi >> 3;
    lo ^= lo >> 35;
    lo *= kMx2;
    lo ^= lo >> 28;
    return H128{lo, avalanche3(hi)};
}

// Hash of one little-endian 64-bit key (8-byte input).
PHB_HD H128 hash_u64(uint64_t key) { return len4to8((uint32_t)key, (uint32_t)(key >> 32), 8); }

// 9..16 bytes given as the first and the last 8 bytes.
PHB_HD H128 len9to16(uint64_t first8, uint64_t last8, uint32_t len) {
    uint64_t bfl = sec64(32) ^ sec64(40);
    uint64_t bfh = sec64(48) ^ sec64(56);
    uint64_t a = first8 ^ last8 ^ bfl;
    uint64_t mlo = a * kP64_1, mhi = mulhi64(a, kP64_1);
    mlo += (uint64_t)(len - 1) << 54;
    uint64_t h2 = last8 ^ bfh;
    mhi += h2 + (uint64_t)(uint32_t)h2 * (kP32_2 - 1);
    mlo ^= bswap64(mhi);
    uint64_t rlo = mlo * kP64_2, rhi = mulhi64(mlo, kP64_2);
    rhi += mhi * kP64_2;
    return H128{avalanche3(rlo), avalanche3(rhi)};
}

// Hash of a 16-byte input given as two little-endian words.
PHB_HD H128 hash_16(uint64_t w0, uint64_t w1) { return len9to16(w0, w1, 16); }

// Byte access to an input that may be unaligned.  The hash below reads its input
// through any type with the same three members (b: one byte, r32 / r64: a little-
// endian word at any byte offset); the kernels also pass a shared-memory stage.
struct ByteSrc {
    const uint8_t *p;
    PHB_HD uint8_t b(size_t i) const { return p[i]; }
    PHB_HD uint64_t r64(size_t i) const {
        uint64_t v = 0;
        for (int k = 7; k >= 0; k--) v = (v << 8) | p[i + k];
        return v;
    }
    PHB_HD uint32_t r32(size_t i) const {
        uint32_t v = 0;
        for (int k = 3; k >= 0; k--) v = (v << 8) | p[i + k];
        return v;
    }
};

template <class Src>
PHB_HD uint64_t mix16(const Src &s, size_t i, unsigned soff) {
    return fold64(s.r64(i) ^ sec64(soff), s.r64(i + 8) ^ sec64(soff + 8));
}

template <class Src>
PHB_HD void mix32(uint64_t &alo, uint64_t &ahi, const Src &s, size_t a, size_t b, unsigned soff) {
    alo += mix16(s, a, soff);
    alo ^= s.r64(b) + s.r64(b + 8);
    ahi += mix16(s, b, soff + 16);
    ahi ^= s.r64(a) + s.r64(a + 8);
}

PHB_HD H128 finish_mid(uint64_t alo, uint64_t ahi, size_t len) {
    uint64_t lo = alo + ahi;
    uint64_t hi = alo * kP64_1 + ahi * kP64_4 + (uint64_t)len * kP64_2;
    return H128{avalanche3(lo), 0 - avalanche3(hi)};
}

template <class Src>
PHB_HD void accumulate_stripe(uint64_t acc[8], const Src &s, size_t i, unsigned soff) {
    for (int j = 0; j < 8; j++) {
        uint64_t v = s.r64(i + 8 * j);
        uint64_t k = v ^ sec64(soff + 8 * j);
        acc[j ^ 1] += v;
        acc[j] += (uint64_t)(uint32_t)k * (k >> 32);
    }
}

PHB_HD uint64_t merge(const uint64_t acc[8], unsigned soff, uint64_t start) {
    uint64_t r = start;
    for (int j = 0; j < 4; j++) r += fold64(acc[2 * j] ^ sec64(soff + 16 * j), acc[2 * j + 1] ^ sec64(soff + 16 * j + 8));
    return avalanche3(r);
}

// XXH3-128 (seed 0) of an arbitrary byte string read through s.
template <class Src>
PHB_HD H128 hash_src(const Src &s, size_t len) {
    if (len == 0) return H128{avalanche64(sec64(64) ^ sec64(72)), avalanche64(sec64(80) ^ sec64(88))};
    if (len <= 3) {
        uint32_t cl = ((uint32_t)s.b(0) << 16) | ((uint32_t)s.b(len >> 1) << 24) | (uint32_t)s.b(len - 1) |
                      ((uint32_t)len << 8);
        uint32_t sw = bswap32(cl);
        uint32_t ch = (sw << 13) | (sw >> 19);
        uint64_t bl = (uint64_t)(sec32(0) ^ sec32(4));
        uint64_t bh = (uint64_t)(sec32(8) ^ sec32(12));
        return H128{avalanche64((uint64_t)cl ^ bl), avalanche64((uint64_t)ch ^ bh)};
    }
    if (len <= 8) return len4to8(s.r32(0), s.r32(len - 4), (uint32_t)len);
    if (len <= 16) return len9to16(s.r64(0), s.r64(len - 8), (uint32_t)len);
    if (len <= 128) {
        uint64_t alo = (uint64_t)len * kP64_1, ahi = 0;
        if (len > 32) {
            if (len > 64) {
                if (len > 96) mix32(alo, ahi, s, 48, len - 64, 96);
                mix32(alo, ahi, s, 32, len - 48, 64);
            }
            mix32(alo, ahi, s, 16, len - 32, 32);
        }
        mix32(alo, ahi, s, 0, len - 16, 0);
        return finish_mid(alo, ahi, len);
    }
    if (len <= 240) {
        uint64_t alo = (uint64_t)len * kP64_1, ahi = 0;
        size_t rounds = len / 32;
        for (size_t r = 0; r < 4; r++) mix32(alo, ahi, s, 32 * r, 32 * r + 16, (unsigned)(32 * r));
        alo = avalanche3(alo);
        ahi = avalanche3(ahi);
        for (size_t r = 4; r < rounds; r++) mix32(alo, ahi, s, 32 * r, 32 * r + 16, (unsigned)(3 + 32 * (r - 4)));
        // Last 32 bytes with the secret window 136 - 17 - 16 and a negated (zero) seed.
        mix32(alo, ahi, s, len - 16, len - 32, 103);
        return finish_mid(alo, ahi, len);
    }
    uint64_t acc[8] = {kP32_3, kP64_1, kP64_2, kP64_3, kP64_4, kP32_2, kP64_5, kP32_1};
    const size_t stripes = (192 - 64) / 8;  // 16 stripes of 64 bytes per block
    const size_t block = 64 * stripes;
    size_t blocks = (len - 1) / block;
    for (size_t bk = 0; bk < blocks; bk++) {
        for (size_t st = 0; st < stripes; st++) accumulate_stripe(acc, s, bk * block + st * 64, (unsigned)(st * 8));
        for (int j = 0; j < 8; j++) {
            uint64_t a = acc[j];
            a ^= a >> 47;
            a ^= sec64(128 + 8 * j);
            acc[j] = a * kP32_1;
        }
    }
    size_t last = ((len - 1) - block * blocks) / 64;
    for (size_t st = 0; st < last; st++) accumulate_stripe(acc, s, blocks * block + st * 64, (unsigned)(st * 8));
    accumulate_stripe(acc, s, len - 64, 192 - 64 - 7);
    return H128{merge(acc, 11, (uint64_t)len * kP64_1), merge(acc, 192 - 64 - 11, ~((uint64_t)len * kP64_2))};
}

// XXH3-128 (seed 0) of an arbitrary byte string.
PHB_HD H128 hash_bytes(const uint8_t *data, size_t len) { return hash_src(ByteSrc{data}, len); }

}  // namespace xxh3

PHB_HD Key4 key_from_hash(xxh3::H128 h) {
    return Key4{(uint32_t)h.lo, (uint32_t)(h.lo >> 32), (uint32_t)h.hi, (uint32_t)(h.hi >> 32)};
}

// ---------------------------------------------------------------- key mapping

PHB_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// key_mapping.glsl:43-45
PHB_HD uint32_t partition_of(uint32_t partitioner, uint32_t partitions) { return mulhi32(partitioner, partitions); }

// key_mapping.glsl:34-41 (32-bit wrapping sum, as the build stages compute it).
PHB_HD uint32_t bucket_of(uint32_t bucketer, uint32_t f_lo, uint32_t f_hi, uint32_t t) {
    return (mulhi32(f_lo, t) + mulhi32(f_hi, 0xFFFFFFFFu - t)) >> 16;
}
PHB_HD uint32_t bucket_of(uint32_t bucketer, const uint32_t *fulcs) {
    uint64_t z = (uint64_t)bucketer * (kFulcrums - 1);
    uint32_t idx = (uint32_t)(z >> 32), t = (uint32_t)z;
    return bucket_of(bucketer, fulcs[idx], fulcs[idx + 1], t);
}

// mphf.hpp:42-49 (64-bit sum, as queries compute it).
PHB_HD uint64_t bucket_of_query(uint32_t bucketer, const uint32_t *fulcs) {
    uint64_t z = (uint64_t)bucketer * (kFulcrums - 1);
    uint64_t idx = z >> 32, part = z & 0xFFFFFFFFULL;
    uint64_t v1 = ((uint64_t)fulcs[idx] * part) >> 32;
    uint64_t v2 = ((uint64_t)fulcs[idx + 1] * (0xFFFFFFFFULL - part)) >> 32;
    return (v1 + v2) >> 16;
}

// hashing.glsl:11-17: one round of the 32-bit mixer after the xor.
PHB_HD uint32_t mix32(uint32_t x) {
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    return (x >> 16) ^ x;
}

// search.comp:31-33 / mphf.hpp:36: hash(lower1, hash(lower2, k)) >> 1.
PHB_HD uint32_t pilot_hash(uint32_t lower1, uint32_t lower2, uint32_t k) { return mix32(lower1 ^ mix32(lower2 ^ k)) >> 1; }

// Query position (mphf.hpp:32-40): fastmod there computes exact a / d and a % d;
// for a partition of one key its fastdiv yields 0, which cannot change the slot.
PHB_HD uint32_t slot_of(uint32_t pilot, uint32_t lower1, uint32_t lower2, uint32_t ps) {
    uint32_t k = ps > 1 ? pilot / ps : 0;
    uint32_t h = pilot_hash(lower1, lower2, k);
    return (h + pilot) % ps;
}

}  // namespace phobicb200
