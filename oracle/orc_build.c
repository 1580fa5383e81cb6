/*
 * Oracle (test infrastructure only): CPU restatement of the PHOBIC-GPU
 * construction pipeline.  Each function names the reference lines it follows.
 * The stage structure is the reference's; the loops are reorganised for a CPU
 * (partition-first, OpenMP over partitions) without changing any result.
 *
 * Canonical choices where the reference is nondeterministic or undefined:
 *   - keys of one bucket keep their input order (the reference's order comes
 *     from global atomicAdd, shaders/bucket_sizes.comp:28); pilots never
 *     depend on this order;
 *   - the pilot of an empty bucket is 0 (the reference leaves it unwritten,
 *     shaders/search.comp:170-174);
 *   - a bucket of more than 256 keys, a partition above the search bitmap
 *     capacity, a bucket id >= buckets, duplicate keys and an exhausted pilot
 *     counter are reported as errors (the reference overruns or spins).
 */
#include "orc.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define DUP_CHECK_AT 256u /* pilot counter at which a bucket is checked for duplicate keys */

static inline uint32_t hi32mul(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

/* key_mapping.glsl:43-45 */
uint32_t orc_partition_of(uint32_t partitioner, uint32_t partitions) { return hi32mul(partitioner, partitions); }

/* key_mapping.glsl:34-41: fulcrum interpolation with 32-bit wrapping arithmetic. */
uint32_t orc_bucket_of(uint32_t bucketer, const uint32_t *fulcs) {
    uint64_t z = (uint64_t)bucketer * (ORC_FULCS - 1);
    uint32_t idx = (uint32_t)(z >> 32);
    uint32_t t = (uint32_t)z;
    uint32_t v1 = hi32mul(fulcs[idx], t);
    uint32_t v2 = hi32mul(fulcs[idx + 1], 0xFFFFFFFFu - t);
    return (v1 + v2) >> 16;
}

/* hashing.glsl:11-17 without the leading xor. */
static inline uint32_t mix32(uint32_t x) {
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    return (x >> 16) ^ x;
}

/* search.comp:31-33: hash(lower1, hash(lower2, k)) >> 1. */
uint32_t orc_pilot_hash(uint32_t lower1, uint32_t lower2, uint32_t k) { return mix32(lower1 ^ mix32(lower2 ^ k)) >> 1; }

/* mphf_config.h:26-34 (ceil) and :36-42 (round). */
uint32_t orc_buckets_per_partition(double lambda, uint32_t partition_size, int use_round) {
    double q = (double)partition_size / lambda;
    return use_round ? (uint32_t)round(q) : (uint32_t)ceil(q);
}

/* bucketers.h:20-50 */
static double bucket_rel(int bucketer, double c, double x) {
    switch (bucketer) {
    case 1: return x;
    case 2: return x < 0.6 ? x / 0.6 * 0.3 : 0.3 + (x - 0.6) / 0.4 * 0.7;
    default: return (x + (1.0 - x) * log(1.0 - x)) * (1.0 - c) + c * x;
    }
}

/* mphf_config.h:44-55 with OptBucketer::init (bucketers.h:28-30). */
void orc_fulcrums(int bucketer, double lambda, uint32_t partition_size, uint32_t buckets, uint32_t *fulcs) {
    double c = 0.2 * lambda / sqrt((double)partition_size);
    uint32_t top = buckets << 16;
    fulcs[0] = 0;
    for (uint32_t xi = 1; xi < ORC_FULCS - 1; xi++) {
        double x = (double)xi / (double)(ORC_FULCS - 1);
        double y = bucket_rel(bucketer, c, x);
        fulcs[xi] = (uint32_t)(y * (double)top);
    }
    fulcs[ORC_FULCS - 1] = top;
}

/* mphf_config.h:61-64 and search.comp:21: the search bitmap holds
 * (1.5 P / 32) words.  At least one word is provided. */
uint32_t orc_max_partition_size(uint32_t partition_size) {
    uint32_t words = (partition_size + partition_size / 2) / 32;
    return 32 * (words ? words : 1);
}

/* ------------------------------------------------------------------ hashing */

static inline void key_words(orc_u128 h, uint32_t *out) {
    out[0] = (uint32_t)h.lo;
    out[1] = (uint32_t)(h.lo >> 32);
    out[2] = (uint32_t)h.hi;
    out[3] = (uint32_t)(h.hi >> 32);
}

void orc_hash_u64(const uint64_t *keys, uint64_t n, uint32_t *keys4, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        orc_u128 h;
        orc_xxh3_128(&keys[i], 8, 0, &h);
        key_words(h, keys4 + 4 * i);
    }
}

void orc_hash_pairs(const uint64_t *pairs, uint64_t n, uint32_t *keys4, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        orc_u128 h;
        orc_xxh3_128(&pairs[2 * i], 16, 0, &h);
        key_words(h, keys4 + 4 * i);
    }
}

/* hasher.hpp:59-65: a Key hashed again as its 16 raw bytes. */
void orc_hash_keys16(const uint32_t *in4, uint64_t n, uint32_t *keys4, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        orc_u128 h;
        orc_xxh3_128(&in4[4 * i], 16, 0, &h);
        key_words(h, keys4 + 4 * i);
    }
}

void orc_hash_bytes(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint32_t *keys4, int threads) {
#pragma omp parallel for schedule(dynamic, 4096) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        orc_u128 h;
        orc_xxh3_128(bytes + offsets[i], (size_t)(offsets[i + 1] - offsets[i]), 0, &h);
        key_words(h, keys4 + 4 * i);
    }
}

void orc_splitmix64(uint64_t seed, uint64_t start, uint64_t n, uint64_t *out, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t z = seed + (start + (uint64_t)i + 1) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        out[i] = z ^ (z >> 31);
    }
}

/* ------------------------------------------------------------------ search */

typedef struct {
    uint64_t *occ;     /* occupied slots; bits [ps, ps+64) mirror [0, 64) */
    uint64_t *scratch; /* duplicate-position detection */
    uint32_t *h;       /* positions of the current bucket */
} search_ws;

static inline uint64_t window64(const uint64_t *occ, uint32_t x) {
    uint32_t w = x >> 6, sh = x & 63;
    return sh ? (occ[w] >> sh) | (occ[w + 1] << (64 - sh)) : occ[w];
}

static inline int occ_bit(const uint64_t *occ, uint32_t q) { return (int)((occ[q >> 6] >> (q & 63)) & 1); }

static inline void occ_set(uint64_t *occ, uint32_t q, uint32_t ps) {
    occ[q >> 6] |= 1ULL << (q & 63);
    if (q < 64) {
        uint32_t m = q + ps;
        occ[m >> 6] |= 1ULL << (m & 63);
    }
}

/* Smallest o in [0, ps) with every (h_i + o) mod ps free (search.comp:72-103
 * under lockstep execution).  Returns ps if there is none. */
static uint32_t first_offset(const search_ws *ws, uint32_t s, uint32_t ps, int naive, uint64_t *probes,
                             uint64_t *key_probes) {
    if (naive) {
        for (uint32_t o = 0; o < ps; o++) {
            uint32_t i = 0;
            for (; i < s; i++) {
                uint32_t pos = ws->h[i] + o;
                if (pos >= ps) pos -= ps;
                if (occ_bit(ws->occ, pos)) break;
            }
            if (i == s) return o;
        }
        return ps;
    }
    for (uint32_t o0 = 0; o0 < ps; o0 += 64) {
        uint64_t bad = 0;
        (*probes)++;
        for (uint32_t i = 0; i < s && bad != ~0ULL; i++) {
            uint32_t x = ws->h[i] + o0;
            if (x >= ps) x -= ps;
            bad |= window64(ws->occ, x);
            (*key_probes)++;
        }
        uint64_t valid = ~bad;
        if (ps - o0 < 64) valid &= (1ULL << (ps - o0)) - 1;
        if (valid) return o0 + (uint32_t)__builtin_ctzll(valid);
    }
    return ps;
}

static int has_duplicate_key(const uint32_t *l1, const uint32_t *l2, uint32_t s) {
    for (uint32_t i = 0; i < s; i++)
        for (uint32_t j = i + 1; j < s; j++)
            if (l1[i] == l1[j] && l2[i] == l2[j]) return 1;
    return 0;
}

/* One bucket: smallest k, then smallest offset (search.comp:105-124). */
static int search_bucket(search_ws *ws, const uint32_t *l1, const uint32_t *l2, uint32_t s, uint32_t ps,
                         uint32_t k_limit, int naive, uint32_t *pilot, orc_stats *st) {
    for (uint32_t k = 0; k < k_limit; k++) {
        if (k == DUP_CHECK_AT && s > 1 && has_duplicate_key(l1, l2, s)) return ORC_ERR_DUPLICATE_KEY;
        for (uint32_t i = 0; i < s; i++) ws->h[i] = orc_pilot_hash(l1[i], l2[i], k) % ps;
        st->hash_evals += s;
        if (s > 1) { /* search.comp:44-70: intra-bucket collision */
            int dup = 0;
            uint32_t i = 0;
            for (; i < s; i++) {
                uint64_t m = 1ULL << (ws->h[i] & 63);
                if (ws->scratch[ws->h[i] >> 6] & m) { dup = 1; break; }
                ws->scratch[ws->h[i] >> 6] |= m;
            }
            for (uint32_t j = 0; j < i + (i < s); j++) ws->scratch[ws->h[j] >> 6] = 0;
            if (dup) { st->k_retries++; continue; }
        }
        uint32_t o = first_offset(ws, s, ps, naive, &st->probe_words, &st->probe_keys);
        if (o < ps) {
            for (uint32_t i = 0; i < s; i++) {
                uint32_t q = ws->h[i] + o;
                if (q >= ps) q -= ps;
                occ_set(ws->occ, q, ps);
            }
            *pilot = o + ps * k;
            if (k > st->max_k) st->max_k = k;
            return ORC_OK;
        }
        st->k_retries++;
    }
    return ORC_ERR_SEARCH_LIMIT;
}

/* ------------------------------------------------------------------ build */

int orc_build(const uint32_t *keys4, uint64_t n, uint32_t P, uint32_t B, const uint32_t *fulcs, uint32_t *pilots,
              uint32_t *part_off, uint32_t *bucket_sizes, uint32_t *histo, uint32_t *perm, uint32_t *sorted_lowers,
              uint32_t max_k, int naive, int threads, orc_stats *stats) {
    orc_stats dummy;
    orc_stats *st = stats ? stats : &dummy;
    memset(st, 0, sizeof(*st));
    st->err_partition = 0xFFFFFFFFu;
    if (P == 0 || B == 0 || B > 65535 || n > 0xFFFFFFFFULL) return ORC_ERR_INVALID;
    if (max_k == 0) max_k = 1u << 20;
    int T = threads > 0 ? threads : omp_get_max_threads();
    uint32_t partitions = (uint32_t)((n + P - 1) / P); /* mphf_builder.h:90 */
    uint32_t cap = orc_max_partition_size(P);
    part_off[0] = 0;
    if (n == 0) return ORC_OK;

    /* Partition id of every key, and the bucket-id range check. */
    uint32_t *pid = (uint32_t *)malloc(n * sizeof(uint32_t));
    int bad_bucket = 0;
#pragma omp parallel for schedule(static) num_threads(T) reduction(| : bad_bucket)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        pid[i] = orc_partition_of(keys4[4 * i], partitions);
        if (orc_bucket_of(keys4[4 * i + 1], fulcs) >= B) bad_bucket = 1;
    }
    if (bad_bucket) {
        free(pid);
        return ORC_ERR_INVALID;
    }

    /* Stable counting sort of key indices by partition (per-thread histograms). */
    uint32_t *hist = (uint32_t *)calloc((size_t)T * partitions, sizeof(uint32_t));
    uint32_t *order = (uint32_t *)malloc(n * sizeof(uint32_t));
#pragma omp parallel num_threads(T)
    {
        int t = omp_get_thread_num();
        uint64_t lo = n * (uint64_t)t / T, hi = n * (uint64_t)(t + 1) / T;
        uint32_t *h = hist + (size_t)t * partitions;
        for (uint64_t i = lo; i < hi; i++) h[pid[i]]++;
#pragma omp barrier
#pragma omp single
        {
            uint64_t run = 0;
            for (uint32_t p = 0; p < partitions; p++) {
                part_off[p] = (uint32_t)run; /* exclusive prefix (mphf_builder.h:254-257) */
                for (int u = 0; u < T; u++) {
                    uint32_t c = hist[(size_t)u * partitions + p];
                    hist[(size_t)u * partitions + p] = (uint32_t)run;
                    run += c;
                }
            }
            part_off[partitions] = (uint32_t)run;
        }
        for (uint64_t i = lo; i < hi; i++) order[h[pid[i]]++] = (uint32_t)i;
    }
    free(hist);
    free(pid);

    for (uint32_t p = 0; p < partitions; p++) {
        uint32_t ps = part_off[p + 1] - part_off[p];
        if (ps > st->max_partition) st->max_partition = ps;
    }
    if (st->max_partition > cap) {
        for (uint32_t p = 0; p < partitions; p++)
            if (part_off[p + 1] - part_off[p] > cap) { st->err_partition = p; break; }
        free(order);
        return ORC_ERR_PARTITION_OVERFLOW;
    }

    int err = ORC_OK;
    uint32_t err_p = 0xFFFFFFFFu;
    uint64_t tot_hash = 0, tot_probe = 0, tot_retry = 0, tot_pkeys = 0;
    uint32_t max_bucket = 0, max_kk = 0;
#pragma omp parallel num_threads(T) reduction(+ : tot_hash, tot_probe, tot_retry, tot_pkeys) reduction(max : max_bucket, max_kk)
    {
        uint32_t *cnt = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *in_bin = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *bstart = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *fill = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *lperm = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *bpil = (uint32_t *)malloc(B * sizeof(uint32_t));
        uint32_t *L1 = (uint32_t *)malloc(cap * sizeof(uint32_t));
        uint32_t *L2 = (uint32_t *)malloc(cap * sizeof(uint32_t));
        uint32_t *kb = (uint32_t *)malloc(cap * sizeof(uint32_t));
        size_t occ_words = (cap + 128) / 64 + 2;
        search_ws ws;
        ws.occ = (uint64_t *)malloc(occ_words * sizeof(uint64_t));
        ws.scratch = (uint64_t *)calloc(occ_words, sizeof(uint64_t));
        ws.h = (uint32_t *)malloc(257 * sizeof(uint32_t));
        uint32_t bins[ORC_BINS], bin_pos[ORC_BINS], bin_key[ORC_BINS];
        orc_stats ls;
        memset(&ls, 0, sizeof(ls));

#pragma omp for schedule(dynamic, 4)
        for (int64_t pp = 0; pp < (int64_t)partitions; pp++) {
            uint32_t p = (uint32_t)pp;
            uint32_t base = part_off[p], ps = part_off[p + 1] - base;
            int perr = ORC_OK;
            /* bucket_sizes.comp:21-35 (ranks in input order) */
            memset(cnt, 0, B * sizeof(uint32_t));
            for (uint32_t i = 0; i < ps; i++) {
                uint32_t b = orc_bucket_of(keys4[4 * (size_t)order[base + i] + 1], fulcs);
                kb[i] = b;
                cnt[b]++;
            }
            if (bucket_sizes) memcpy(bucket_sizes + (size_t)p * B, cnt, B * sizeof(uint32_t));
            for (uint32_t b = 0; b < B; b++) {
                if (cnt[b] > max_bucket) max_bucket = cnt[b];
                if (cnt[b] > ORC_BINS) perr = ORC_ERR_BUCKET_OVERFLOW;
            }
            /* sort_sum.comp:156-225: bin = 256 - size, lane 0 walks buckets B-1..0 */
            memset(bins, 0, sizeof(bins));
            for (int64_t b = (int64_t)B - 1; b >= 0 && perr == ORC_OK; b--) {
                uint32_t s = cnt[b];
                if (s > 0) in_bin[b] = bins[ORC_BINS - s]++;
            }
            uint32_t nonempty = 0;
            if (perr == ORC_OK) {
                if (histo) memcpy(histo + (size_t)p * ORC_BINS, bins, sizeof(bins));
                uint32_t run = 0, krun = 0;
                for (uint32_t i = 0; i < ORC_BINS; i++) {
                    bin_pos[i] = run;
                    bin_key[i] = krun;
                    run += bins[i];
                    krun += bins[i] * (ORC_BINS - i);
                }
                nonempty = run;
                memset(lperm, 0, B * sizeof(uint32_t));
                for (uint32_t b = 0; b < B; b++) {
                    uint32_t s = cnt[b];
                    if (!s) continue;
                    lperm[bin_pos[ORC_BINS - s] + in_bin[b]] = b;
                    bstart[b] = bin_key[ORC_BINS - s] + in_bin[b] * s;
                }
                if (perm) memcpy(perm + (size_t)p * B, lperm, B * sizeof(uint32_t));
                /* redistribute_keys.comp:21-53 (stable within a bucket) */
                memset(fill, 0, B * sizeof(uint32_t));
                for (uint32_t i = 0; i < ps; i++) {
                    uint32_t b = kb[i];
                    uint32_t pos = bstart[b] + fill[b]++;
                    const uint32_t *k4 = keys4 + 4 * (size_t)order[base + i];
                    L1[pos] = k4[2];
                    L2[pos] = k4[3];
                }
                if (sorted_lowers)
                    for (uint32_t i = 0; i < ps; i++) {
                        sorted_lowers[2 * ((size_t)base + i)] = L1[i];
                        sorted_lowers[2 * ((size_t)base + i) + 1] = L2[i];
                    }
                /* search.comp:126-175 */
                uint32_t k_limit = (uint32_t)(0x80000000ULL / (ps ? ps : 1));
                if (k_limit > max_k) k_limit = max_k;
                memset(ws.occ, 0, occ_words * sizeof(uint64_t));
                memset(bpil, 0, B * sizeof(uint32_t));
                for (uint32_t j = 0; j < nonempty && perr == ORC_OK; j++) {
                    uint32_t b = lperm[j], s = cnt[b], st0 = bstart[b];
                    perr = search_bucket(&ws, L1 + st0, L2 + st0, s, ps, k_limit, naive, &bpil[b], &ls);
                }
            }
            for (uint32_t b = 0; b < B; b++) pilots[(size_t)b * partitions + p] = perr == ORC_OK ? bpil[b] : 0;
            if (perr != ORC_OK) {
#pragma omp critical
                {
                    if (p < err_p) {
                        err_p = p;
                        err = perr;
                    }
                }
            }
        }
        tot_hash += ls.hash_evals;
        tot_probe += ls.probe_words;
        tot_retry += ls.k_retries;
        tot_pkeys += ls.probe_keys;
        if (ls.max_k > max_kk) max_kk = ls.max_k;
        free(cnt); free(in_bin); free(bstart); free(fill); free(lperm); free(bpil);
        free(L1); free(L2); free(kb); free(ws.occ); free(ws.scratch); free(ws.h);
    }
    free(order);
    st->hash_evals = tot_hash;
    st->probe_words = tot_probe;
    st->k_retries = tot_retry;
    st->probe_keys = tot_pkeys;
    st->max_bucket = max_bucket;
    st->max_k = max_kk;
    st->err_partition = err_p;
    return err;
}

/* ------------------------------------------------------------------ query */

/* mphf.hpp:42-49: 64-bit form of the bucket mapping used by queries. */
static inline uint64_t query_bucket(uint32_t bucketer, const uint32_t *fulcs) {
    uint64_t z = (uint64_t)bucketer * (ORC_FULCS - 1);
    uint64_t idx = z >> 32, part = z & 0xFFFFFFFFULL;
    uint64_t v1 = ((uint64_t)fulcs[idx] * part) >> 32;
    uint64_t v2 = ((uint64_t)fulcs[idx + 1] * (0xFFFFFFFFULL - part)) >> 32;
    return (v1 + v2) >> 16;
}

/* mphf.hpp:32-40 and :77-86 (fastmod computes exact a / d and a % d; for a
 * partition of one key its fastdiv yields 0, which cannot change the slot). */
void orc_query(const uint32_t *keys4, uint64_t n, uint32_t partitions, uint32_t buckets, const uint32_t *fulcs,
               const uint32_t *pilots, const uint32_t *part_off, uint32_t *out, int threads) {
    (void)buckets;
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const uint32_t *k4 = keys4 + 4 * i;
        uint32_t p = (uint32_t)(((uint64_t)k4[0] * partitions) >> 32);
        uint64_t b = query_bucket(k4[1], fulcs);
        uint32_t pilot = pilots[b * partitions + p];
        uint32_t off = part_off[p], ps = part_off[p + 1] - off;
        uint32_t k = ps > 1 ? pilot / ps : 0;
        uint32_t h = orc_pilot_hash(k4[2], k4[3], k);
        out[i] = off + (uint32_t)(h + pilot) % ps;
    }
}

int orc_is_bijection(const uint32_t *pos, uint64_t n) {
    uint8_t *seen = (uint8_t *)calloc(n ? n : 1, 1);
    int ok = 1;
    for (uint64_t i = 0; i < n && ok; i++) {
        if (pos[i] >= n || seen[pos[i]]) ok = 0;
        else seen[pos[i]] = 1;
    }
    free(seen);
    return ok;
}
