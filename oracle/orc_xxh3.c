/*
 * Oracle (test infrastructure only): XXH3-128 restated in plain C.
 *
 * The reference hashes every key with `XXH128(data, len, 0)` from the xxHash
 * library (include/phobicGpu/hasher.hpp:33-66), pulled in through the git
 * submodule external/xxHash (branch `release`, .gitmodules:7-10).  That
 * submodule is empty in the reference checkout, so the pinned commit is
 * unknown; XXH3-128 output has been frozen since xxHash v0.8.0, and the
 * golden vectors under tests/golden/ were produced by the `xxhash` Python
 * module built on libxxhash 0.8.2.  This file restates the published XXH3
 * algorithm (xxHash specification, "XXH3" section) for seed 0 and any seed
 * that does not require a derived secret (all inputs <= 240 bytes, and long
 * inputs with seed 0).
 *
 * Only tests/, the golden-vector generator and bench.py's CPU baseline load
 * this code, and only as a checker.
 */
#include "orc.h"

#include <string.h>

#define P32_1 0x9E3779B1U
#define P32_2 0x85EBCA77U
#define P32_3 0xC2B2AE3DU
#define P64_1 0x9E3779B185EBCA87ULL
#define P64_2 0xC2B2AE3D27D4EB4FULL
#define P64_3 0x165667B19E3779F9ULL
#define P64_4 0x85EBCA77C2B2AE63ULL
#define P64_5 0x27D4EB2F165667C5ULL
#define PMX_1 0x165667919E3779F9ULL
#define PMX_2 0x9FB21C651E98DF25ULL

/* Default 192-byte secret of XXH3 (xxHash specification). */
static const uint8_t kSecret[192] = {
    0xb8, 0xfe, 0x6c, 0x39, 0x23, 0xa4, 0x4b, 0xbe, 0x7c, 0x01, 0x81, 0x2c, 0xf7, 0x21, 0xad, 0x1c,
    0xde, 0xd4, 0x6d, 0xe9, 0x83, 0x90, 0x97, 0xdb, 0x72, 0x40, 0xa4, 0xa4, 0xb7, 0xb3, 0x67, 0x1f,
    0xcb, 0x79, 0xe6, 0x4e, 0xcc, 0xc0, 0xe5, 0x78, 0x82, 0x5a, 0xd0, 0x7d, 0xcc, 0xff, 0x72, 0x21,
    0xb8, 0x08, 0x46, 0x74, 0xf7, 0x43, 0x24, 0x8e, 0xe0, 0x35, 0x90, 0xe6, 0x81, 0x3a, 0x26, 0x4c,
    0x3c, 0x28, 0x52, 0xbb, 0x91, 0xc3, 0x00, 0xcb, 0x88, 0xd0, 0x65, 0x8b, 0x1b, 0x53, 0x2e, 0xa3,
    0x71, 0x64, 0x48, 0x97, 0xa2, 0x0d, 0xf9, 0x4e, 0x38, 0x19, 0xef, 0x46, 0xa9, 0xde, 0xac, 0xd8,
    0xa8, 0xfa, 0x76, 0x3f, 0xe3, 0x9c, 0x34, 0x3f, 0xf9, 0xdc, 0xbb, 0xc7, 0xc7, 0x0b, 0x4f, 0x1d,
    0x8a, 0x51, 0xe0, 0x4b, 0xcd, 0xb4, 0x59, 0x31, 0xc8, 0x9f, 0x7e, 0xc9, 0xd9, 0x78, 0x73, 0x64,
    0xea, 0xc5, 0xac, 0x83, 0x34, 0xd3, 0xeb, 0xc3, 0xc5, 0x81, 0xa0, 0xff, 0xfa, 0x13, 0x63, 0xeb,
    0x17, 0x0d, 0xdd, 0x51, 0xb7, 0xf0, 0xda, 0x49, 0xd3, 0x16, 0x55, 0x26, 0x29, 0xd4, 0x68, 0x9e,
    0x2b, 0x16, 0xbe, 0x58, 0x7d, 0x47, 0xa1, 0xfc, 0x8f, 0xf8, 0xb8, 0xd1, 0x7a, 0xd0, 0x31, 0xce,
    0x45, 0xcb, 0x3a, 0x8f, 0x95, 0x16, 0x04, 0x28, 0xaf, 0xd7, 0xfb, 0xca, 0xbb, 0x4b, 0x40, 0x7e,
};

static inline uint64_t rd64(const uint8_t *p) {
    uint64_t v;
    memcpy(&v, p, 8); /* x86-64 is little endian, as the specification reads */
    return v;
}
static inline uint32_t rd32(const uint8_t *p) {
    uint32_t v;
    memcpy(&v, p, 4);
    return v;
}
static inline uint32_t bswap32(uint32_t x) { return __builtin_bswap32(x); }
static inline uint64_t bswap64(uint64_t x) { return __builtin_bswap64(x); }
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

static inline orc_u128 mul64to128(uint64_t a, uint64_t b) {
    unsigned __int128 p = (unsigned __int128)a * b;
    orc_u128 r = {(uint64_t)p, (uint64_t)(p >> 64)};
    return r;
}
static inline uint64_t mul128_fold64(uint64_t a, uint64_t b) {
    orc_u128 p = mul64to128(a, b);
    return p.lo ^ p.hi;
}
static inline uint64_t xorshift64(uint64_t v, int s) { return v ^ (v >> s); }

static inline uint64_t xxh64_avalanche(uint64_t h) {
    h ^= h >> 33;
    h *= P64_2;
    h ^= h >> 29;
    h *= P64_3;
    h ^= h >> 32;
    return h;
}
static inline uint64_t xxh3_avalanche(uint64_t h) {
    h = xorshift64(h, 37);
    h *= PMX_1;
    return xorshift64(h, 32);
}

static orc_u128 len_1to3(const uint8_t *in, size_t len, const uint8_t *sec, uint64_t seed) {
    uint8_t c1 = in[0], c2 = in[len >> 1], c3 = in[len - 1];
    uint32_t cl = ((uint32_t)c1 << 16) | ((uint32_t)c2 << 24) | ((uint32_t)c3 << 0) | ((uint32_t)len << 8);
    uint32_t ch = rotl32(bswap32(cl), 13);
    uint64_t bfl = (uint64_t)(rd32(sec) ^ rd32(sec + 4)) + seed;
    uint64_t bfh = (uint64_t)(rd32(sec + 8) ^ rd32(sec + 12)) - seed;
    orc_u128 r = {xxh64_avalanche((uint64_t)cl ^ bfl), xxh64_avalanche((uint64_t)ch ^ bfh)};
    return r;
}

static orc_u128 len_4to8(const uint8_t *in, size_t len, const uint8_t *sec, uint64_t seed) {
    seed ^= (uint64_t)bswap32((uint32_t)seed) << 32;
    uint32_t lo = rd32(in), hi = rd32(in + len - 4);
    uint64_t in64 = (uint64_t)lo + ((uint64_t)hi << 32);
    uint64_t bitflip = (rd64(sec + 16) ^ rd64(sec + 24)) + seed;
    uint64_t keyed = in64 ^ bitflip;
    orc_u128 m = mul64to128(keyed, P64_1 + ((uint64_t)len << 2));
    m.hi += (m.lo << 1);
    m.lo ^= (m.hi >> 3);
    m.lo = xorshift64(m.lo, 35);
    m.lo *= PMX_2;
    m.lo = xorshift64(m.lo, 28);
    m.hi = xxh3_avalanche(m.hi);
    return m;
}

static orc_u128 len_9to16(const uint8_t *in, size_t len, const uint8_t *sec, uint64_t seed) {
    uint64_t bfl = (rd64(sec + 32) ^ rd64(sec + 40)) - seed;
    uint64_t bfh = (rd64(sec + 48) ^ rd64(sec + 56)) + seed;
    uint64_t ilo = rd64(in);
    uint64_t ihi = rd64(in + len - 8);
    orc_u128 m = mul64to128(ilo ^ ihi ^ bfl, P64_1);
    m.lo += (uint64_t)(len - 1) << 54;
    ihi ^= bfh;
    m.hi += ihi + (uint64_t)(uint32_t)ihi * (uint64_t)(P32_2 - 1);
    m.lo ^= bswap64(m.hi);
    orc_u128 h = mul64to128(m.lo, P64_2);
    h.hi += m.hi * P64_2;
    h.lo = xxh3_avalanche(h.lo);
    h.hi = xxh3_avalanche(h.hi);
    return h;
}

static inline uint64_t mix16(const uint8_t *in, const uint8_t *sec, uint64_t seed) {
    return mul128_fold64(rd64(in) ^ (rd64(sec) + seed), rd64(in + 8) ^ (rd64(sec + 8) - seed));
}

static inline orc_u128 mix32(orc_u128 acc, const uint8_t *a, const uint8_t *b, const uint8_t *sec, uint64_t seed) {
    acc.lo += mix16(a, sec, seed);
    acc.lo ^= rd64(b) + rd64(b + 8);
    acc.hi += mix16(b, sec + 16, seed);
    acc.hi ^= rd64(a) + rd64(a + 8);
    return acc;
}

static orc_u128 finish_mid(orc_u128 acc, size_t len, uint64_t seed) {
    orc_u128 h;
    h.lo = acc.lo + acc.hi;
    h.hi = acc.lo * P64_1 + acc.hi * P64_4 + ((uint64_t)len - seed) * P64_2;
    h.lo = xxh3_avalanche(h.lo);
    h.hi = 0 - xxh3_avalanche(h.hi);
    return h;
}

static orc_u128 len_17to128(const uint8_t *in, size_t len, const uint8_t *sec, uint64_t seed) {
    orc_u128 acc = {(uint64_t)len * P64_1, 0};
    if (len > 32) {
        if (len > 64) {
            if (len > 96) acc = mix32(acc, in + 48, in + len - 64, sec + 96, seed);
            acc = mix32(acc, in + 32, in + len - 48, sec + 64, seed);
        }
        acc = mix32(acc, in + 16, in + len - 32, sec + 32, seed);
    }
    acc = mix32(acc, in, in + len - 16, sec, seed);
    return finish_mid(acc, len, seed);
}

static orc_u128 len_129to240(const uint8_t *in, size_t len, const uint8_t *sec, uint64_t seed) {
    size_t rounds = len / 32;
    orc_u128 acc = {(uint64_t)len * P64_1, 0};
    for (size_t i = 0; i < 4; i++) acc = mix32(acc, in + 32 * i, in + 32 * i + 16, sec + 32 * i, seed);
    acc.lo = xxh3_avalanche(acc.lo);
    acc.hi = xxh3_avalanche(acc.hi);
    for (size_t i = 4; i < rounds; i++)
        acc = mix32(acc, in + 32 * i, in + 32 * i + 16, sec + 3 + 32 * (i - 4), seed);
    /* last 32 bytes, secret window ends 17 bytes before the 136-byte minimum */
    acc = mix32(acc, in + len - 16, in + len - 32, sec + 136 - 17 - 16, 0 - seed);
    return finish_mid(acc, len, seed);
}

static void accumulate512(uint64_t acc[8], const uint8_t *in, const uint8_t *sec) {
    for (int i = 0; i < 8; i++) {
        uint64_t v = rd64(in + 8 * i);
        uint64_t k = v ^ rd64(sec + 8 * i);
        acc[i ^ 1] += v;
        acc[i] += (uint64_t)(uint32_t)k * (k >> 32);
    }
}

static void scramble(uint64_t acc[8], const uint8_t *sec) {
    for (int i = 0; i < 8; i++) {
        uint64_t a = acc[i];
        a = xorshift64(a, 47);
        a ^= rd64(sec + 8 * i);
        a *= P32_1;
        acc[i] = a;
    }
}

static uint64_t merge_accs(const uint64_t acc[8], const uint8_t *sec, uint64_t start) {
    uint64_t r = start;
    for (int i = 0; i < 4; i++) r += mul128_fold64(acc[2 * i] ^ rd64(sec + 16 * i), acc[2 * i + 1] ^ rd64(sec + 16 * i + 8));
    return xxh3_avalanche(r);
}

static orc_u128 hash_long(const uint8_t *in, size_t len, const uint8_t *sec, size_t secsz) {
    uint64_t acc[8] = {P32_3, P64_1, P64_2, P64_3, P64_4, P32_2, P64_5, P32_1};
    size_t stripes_per_block = (secsz - 64) / 8;
    size_t block_len = 64 * stripes_per_block;
    size_t nb_blocks = (len - 1) / block_len;
    for (size_t b = 0; b < nb_blocks; b++) {
        for (size_t s = 0; s < stripes_per_block; s++) accumulate512(acc, in + b * block_len + s * 64, sec + s * 8);
        scramble(acc, sec + secsz - 64);
    }
    size_t nb_stripes = ((len - 1) - block_len * nb_blocks) / 64;
    for (size_t s = 0; s < nb_stripes; s++) accumulate512(acc, in + nb_blocks * block_len + s * 64, sec + s * 8);
    accumulate512(acc, in + len - 64, sec + secsz - 64 - 7);
    orc_u128 h;
    h.lo = merge_accs(acc, sec + 11, (uint64_t)len * P64_1);
    h.hi = merge_accs(acc, sec + secsz - 64 - 11, ~((uint64_t)len * P64_2));
    return h;
}

int orc_xxh3_128(const void *data, size_t len, uint64_t seed, orc_u128 *out) {
    const uint8_t *in = (const uint8_t *)data;
    if (len == 0) {
        out->lo = xxh64_avalanche(seed ^ rd64(kSecret + 64) ^ rd64(kSecret + 72));
        out->hi = xxh64_avalanche(seed ^ rd64(kSecret + 80) ^ rd64(kSecret + 88));
        return 0;
    }
    if (len <= 3) { *out = len_1to3(in, len, kSecret, seed); return 0; }
    if (len <= 8) { *out = len_4to8(in, len, kSecret, seed); return 0; }
    if (len <= 16) { *out = len_9to16(in, len, kSecret, seed); return 0; }
    if (len <= 128) { *out = len_17to128(in, len, kSecret, seed); return 0; }
    if (len <= 240) { *out = len_129to240(in, len, kSecret, seed); return 0; }
    if (seed != 0) return -1; /* a seeded long hash needs a derived secret: not on the path */
    *out = hash_long(in, len, kSecret, sizeof(kSecret));
    return 0;
}
