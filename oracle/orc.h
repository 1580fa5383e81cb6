/*
 * Oracle for the PHOBIC MPHF construction path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, CPU restatement of the reference's construction pipeline:
 *   - initial hash        include/phobicGpu/hasher.hpp:30-67 (XXH128, seed 0)
 *   - fulcrum table        include/phobicGpu/mphf_config.h:26-55, bucketers.h:20-50
 *   - key mapping          shaders/key_mapping.glsl:9-49
 *   - bucket sizes         shaders/bucket_sizes.comp:21-35
 *   - bucket sort          shaders/sort_sum.comp:141-226
 *   - partition offsets    shaders/prefix_sum.comp, prefix_sum_offset.comp,
 *                          apply_partition_offset.comp:9-18,
 *                          include/phobicGpu/mphf_builder.h:254-257
 *   - redistribution       shaders/redistribute_keys.comp:21-53
 *   - pilot search         shaders/search.comp:31-175, shaders/hashing.glsl:11-17
 *   - query                include/phobicGpu/mphf.hpp:32-49,77-86
 *
 * It is the checker for the CUDA path: only tests/, the golden-vector
 * generator under tests/golden/ and bench.py's CPU-baseline leg load it.
 * Nothing in the product links against it.
 */
#ifndef PHOBIC_ORACLE_H
#define PHOBIC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t lo;
    uint64_t hi;
} orc_u128;

enum {
    ORC_OK = 0,
    ORC_ERR_INVALID = 1,
    ORC_ERR_BUCKET_OVERFLOW = 3,
    ORC_ERR_PARTITION_OVERFLOW = 4,
    ORC_ERR_SEARCH_LIMIT = 5,
    ORC_ERR_DUPLICATE_KEY = 8,
};

#define ORC_FULCS 2048
#define ORC_BINS 256

/* XXH3-128 of `len` bytes (seed must be 0 for len > 240). Returns 0 on success. */
int orc_xxh3_128(const void *data, size_t len, uint64_t seed, orc_u128 *out);

/* Initial hash into 4-word Keys {partitioner, bucketer, lower1, lower2}
 * (hasher.hpp:7-20,42-48): words = [lo32(low64), hi32(low64), lo32(high64), hi32(high64)]. */
void orc_hash_u64(const uint64_t *keys, uint64_t n, uint32_t *keys4, int threads);
void orc_hash_pairs(const uint64_t *pairs, uint64_t n, uint32_t *keys4, int threads);
void orc_hash_keys16(const uint32_t *in4, uint64_t n, uint32_t *keys4, int threads);
void orc_hash_bytes(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint32_t *keys4, int threads);

/* MPHFconfig arithmetic (mphf_config.h:26-64). bucketer: 0 = Opt, 1 = Uniform, 2 = Skew.
 * use_round selects the Bucketer* constructor's round() instead of ceil(). */
uint32_t orc_buckets_per_partition(double lambda, uint32_t partition_size, int use_round);
void orc_fulcrums(int bucketer, double lambda, uint32_t partition_size, uint32_t buckets, uint32_t *fulcs);
uint32_t orc_max_partition_size(uint32_t partition_size);

/* Key mapping (key_mapping.glsl:34-49). */
uint32_t orc_partition_of(uint32_t partitioner, uint32_t partitions);
uint32_t orc_bucket_of(uint32_t bucketer, const uint32_t *fulcs);
uint32_t orc_pilot_hash(uint32_t lower1, uint32_t lower2, uint32_t k);

typedef struct {
    uint64_t hash_evals;    /* hash evaluations made by the search (all k) */
    uint64_t probe_words;   /* 64-offset windows tested (one per window, whatever the bucket size) */
    uint64_t k_retries;     /* pilot-counter increments over all buckets */
    uint32_t max_bucket;    /* largest bucket */
    uint32_t max_partition; /* largest partition */
    uint32_t max_k;         /* largest pilot counter used */
    uint32_t err_partition; /* partition of the first error */
    uint32_t pad;
    uint64_t probe_keys;    /* bitmap probes: one 64-bit window of one key's slot (window64 calls);
                               a window stops taking keys once every offset in it is rejected */
} orc_stats;

/*
 * Whole construction from 4-word Keys.  Outputs (caller-allocated):
 *   pilots[buckets * partitions]      bucket-major: pilots[b * partitions + p]
 *   part_off[partitions + 1]          exclusive prefix of partition sizes, [0] = 0
 * Optional intermediates (NULL to skip):
 *   bucket_sizes[partitions * buckets] key count of bucket b of partition p at [p*buckets + b]
 *   histo[partitions * 256]           sort_sum.comp histogram: bin 256-size
 *   perm[partitions * buckets]        bucket ids in (size desc, index desc) order, unused tail = 0
 *   sorted_lowers[2 * n]              (lower1, lower2) in partition, then search order,
 *                                     keys of one bucket in input order
 * max_k caps the pilot counter (0 = default 1<<20).  naive != 0 tests offsets one at a
 * time exactly as written in search.comp instead of 64-offset windows.
 */
int orc_build(const uint32_t *keys4, uint64_t n, uint32_t partition_size, uint32_t buckets,
              const uint32_t *fulcs, uint32_t *pilots, uint32_t *part_off, uint32_t *bucket_sizes,
              uint32_t *histo, uint32_t *perm, uint32_t *sorted_lowers, uint32_t max_k, int naive,
              int threads, orc_stats *stats);

/* Query (mphf.hpp:77-86) over the raw layout.  out[i] = position of key i. */
void orc_query(const uint32_t *keys4, uint64_t n, uint32_t partitions, uint32_t buckets,
               const uint32_t *fulcs, const uint32_t *pilots, const uint32_t *part_off, uint32_t *out,
               int threads);

/* Returns 1 if out[0..n) is a permutation of [0, n). */
int orc_is_bijection(const uint32_t *pos, uint64_t n);

/* splitmix64 stream (Vigna): x_{i} = seed + (i+1)*0x9E3779B97F4A7C15, then the finalizer. */
void orc_splitmix64(uint64_t seed, uint64_t start, uint64_t n, uint64_t *out, int threads);

#ifdef __cplusplus
}
#endif
#endif
