/*
 * pj_oracle.c -- CPU restatement of the reference's radix-partitioned
 * inner equi-join path (Feng-Jiang28/partitioned_join).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked by the
 * tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, and
 * never by the product library.  The CUDA path in partitioned_join_b200/
 * does not call it and fails loudly when its own extension is missing.
 *
 * Pinning: every function here is checked against golden vectors produced
 * by the reference's own sources compiled in this container
 * (tests/golden/make_golden.py drives oracle/_ref/libref_cpu.so, built by
 * oracle/build_ref.sh from src/hash_functions.cuh, src/int_fastdiv.h and
 * src/inner_join_cpu.hpp); tests/test_oracle_golden.py holds the checks.
 *
 * Each function cites the reference file:line it restates.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* MurmurHash3_x86_32, seed 0, over the key's little-endian bytes.
 * Restates src/hash_functions.cuh:80-119 (body :94-105, tail :108-115 is
 * empty for 4- and 8-byte keys, finalisation :117-118 with fmix32 :47-55).
 * The algorithm itself is Austin Appleby's public-domain MurmurHash3. */
static uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

static uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

static uint32_t murmur_block(uint32_t h1, uint32_t k1)
{
    k1 *= 0xcc9e2d51u;
    k1 = rotl32(k1, 15);
    k1 *= 0x1b873593u;
    h1 ^= k1;
    h1 = rotl32(h1, 13);
    return h1 * 5u + 0xe6546b64u;
}

uint32_t pjo_hash_i32(int32_t key)
{
    uint32_t h = murmur_block(0u, (uint32_t)key);
    h ^= 4u;
    return fmix32(h);
}

uint32_t pjo_hash_i64(int64_t key)
{
    uint64_t u = (uint64_t)key;
    uint32_t h = murmur_block(0u, (uint32_t)(u & 0xffffffffu)); /* first block in memory order */
    h = murmur_block(h, (uint32_t)(u >> 32));
    h ^= 8u;
    return fmix32(h);
}

void pjo_hash_array(const void* keys, int64_t n, int key_bytes, uint32_t* out)
{
    int64_t i;
    if (key_bytes == 4) {
        const int32_t* k = (const int32_t*)keys;
        for (i = 0; i < n; ++i) out[i] = pjo_hash_i32(k[i]);
    } else {
        const int64_t* k = (const int64_t*)keys;
        for (i = 0; i < n; ++i) out[i] = pjo_hash_i64(k[i]);
    }
}

/* ------------------------------------------------------------------------ */
/* Hash-table slot of the reference join: abs((int)h % T), with % the
 * truncating signed remainder that int_fastdiv computes for an unsigned
 * dividend cast to int.  src/hash_join_kernels.cuh:100-101 (build) and
 * :141-142 (probe); src/int_fastdiv.h:118-133,142-145. */
int32_t pjo_ref_slot(uint32_t h, int32_t table_size)
{
    int32_t r = (int32_t)h % table_size;
    return r < 0 ? -r : r;
}

/* ------------------------------------------------------------------------ */
/* Partition digit functions.
 *   mode 0 (reference, raw key bits):
 *     one pass          d = key & (P-1)                 partition_kernels.cuh:168 with num_bit_p2 = 0
 *     two-pass, pass 1  d = ((P1-1) << b2 & key) >> b2  partition_kernels.cuh:168,177,236,244,292
 *     two-pass, pass 2  d = key & (P2-1)                partition_kernels.cuh:380,389,471,479,527
 *   mode 1 (hash bits; the B200 build's robust default, no reference
 *     counterpart): d = top (b1+b2) bits of murmur(key); pass 1 takes the
 *     top b1 bits, pass 2 the next b2 bits.
 * `which` = 0 for the combined digit (p1 * P2 + p2), 1 for pass 1, 2 for pass 2. */
int32_t pjo_digit_i64(int64_t key, uint32_t h, int mode, int b1, int b2, int which)
{
    if (mode == 0) {
        int64_t p1 = (((int64_t)((1 << b1) - 1) << b2) & key) >> b2;
        int64_t p2 = key & (int64_t)((1 << b2) - 1);
        if (which == 1) return (int32_t)p1;
        if (which == 2) return (int32_t)p2;
        return (int32_t)((p1 << b2) | p2);
    } else {
        int D = b1 + b2;
        uint32_t all = D == 0 ? 0u : (h >> (32 - D));
        if (which == 1) return (int32_t)(all >> b2);
        if (which == 2) return (int32_t)(all & ((1u << b2) - 1u));
        return (int32_t)all;
    }
}

void pjo_digits(const void* keys, int64_t n, int key_bytes, int mode, int b1, int b2, int which,
                int32_t* out)
{
    int64_t i;
    for (i = 0; i < n; ++i) {
        int64_t k = key_bytes == 4 ? (int64_t)((const int32_t*)keys)[i] : ((const int64_t*)keys)[i];
        uint32_t h = key_bytes == 4 ? pjo_hash_i32((int32_t)k) : pjo_hash_i64(k);
        out[i] = pjo_digit_i64(k, h, mode, b1, b2, which);
    }
}

/* Digit histogram over a key column: the global result of
 * histogram_pass_one (partition_kernels.cuh:141-194), histogram_pass_two
 * (:329-406) and big_histogram (:86-124), which all count keys per digit. */
void pjo_histogram(const void* keys, int64_t n, int key_bytes, int mode, int b1, int b2,
                   int which, int32_t* counts)
{
    int64_t i;
    int nb = which == 1 ? b1 : which == 2 ? b2 : b1 + b2;
    memset(counts, 0, sizeof(int32_t) * ((size_t)1 << nb));
    for (i = 0; i < n; ++i) {
        int64_t k = key_bytes == 4 ? (int64_t)((const int32_t*)keys)[i] : ((const int64_t*)keys)[i];
        uint32_t h = key_bytes == 4 ? pjo_hash_i32((int32_t)k) : pjo_hash_i64(k);
        counts[pjo_digit_i64(k, h, mode, b1, b2, which)]++;
    }
}

/* ------------------------------------------------------------------------ */
/* inner_join_cpu restated to emit (build_row, probe_row).
 * src/inner_join_cpu.hpp:24-107.  The reference stores the build row as the
 * map value (:52, :85) but emits {key, 0}; this restatement emits the stored
 * row instead, so its key projection equals the reference's output.
 *   unique_keys != 0: std::unordered_map::insert keeps the FIRST row of a
 *     repeated key (:51-53); each probe row matches at most once (:59-75).
 *   unique_keys == 0: std::unordered_multimap, every (build, probe) pair with
 *     equal keys (:83-101).
 * Writes at most `capacity` pairs; returns the total number of pairs.
 * The table is plain open addressing on murmur(key) with a per-key chain of
 * build rows; layout does not affect the result multiset. */
typedef struct {
    int64_t key;
    int32_t head;  /* first build row with this key, -1 = empty slot */
    int32_t tail;
} pjo_slot;

int64_t pjo_inner_join(const void* build_keys, int64_t n_build,
                       const void* probe_keys, int64_t n_probe, int key_bytes,
                       int unique_keys, int32_t* out_build_row, int32_t* out_probe_row,
                       int64_t capacity)
{
    uint64_t cap = 16, mask;
    int64_t i, total = 0;
    pjo_slot* table;
    int32_t* next;
    while (cap < (uint64_t)(2 * n_build + 1)) cap <<= 1;
    mask = cap - 1;
    table = (pjo_slot*)malloc(sizeof(pjo_slot) * cap);
    next = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_build > 0 ? n_build : 1));
    if (!table || !next) {
        free(table);
        free(next);
        return -1;
    }
    for (i = 0; i < (int64_t)cap; ++i) table[i].head = -1;

    for (i = 0; i < n_build; ++i) {
        int64_t k = key_bytes == 4 ? (int64_t)((const int32_t*)build_keys)[i] : ((const int64_t*)build_keys)[i];
        uint32_t h = key_bytes == 4 ? pjo_hash_i32((int32_t)k) : pjo_hash_i64(k);
        uint64_t s = h & mask;
        next[i] = -1;
        for (;;) {
            if (table[s].head < 0) {
                table[s].key = k;
                table[s].head = (int32_t)i;
                table[s].tail = (int32_t)i;
                break;
            }
            if (table[s].key == k) {
                if (!unique_keys) { /* multimap: append, keeps insertion order */
                    next[table[s].tail] = (int32_t)i;
                    table[s].tail = (int32_t)i;
                }
                break; /* unique: unordered_map::insert keeps the first */
            }
            s = (s + 1) & mask;
        }
    }

    for (i = 0; i < n_probe; ++i) {
        int64_t k = key_bytes == 4 ? (int64_t)((const int32_t*)probe_keys)[i] : ((const int64_t*)probe_keys)[i];
        uint32_t h = key_bytes == 4 ? pjo_hash_i32((int32_t)k) : pjo_hash_i64(k);
        uint64_t s = h & mask;
        for (;;) {
            if (table[s].head < 0) break;
            if (table[s].key == k) {
                int32_t r = table[s].head;
                while (r >= 0) {
                    if (total < capacity) {
                        out_build_row[total] = r;
                        out_probe_row[total] = (int32_t)i;
                    }
                    ++total;
                    r = next[r];
                }
                break;
            }
            s = (s + 1) & mask;
        }
    }
    free(table);
    free(next);
    return total;
}

/* Number of output pairs without writing them (the count the reference's
 * main.cu:697-704 takes from the CPU run to size the GPU output). */
int64_t pjo_join_count(const void* build_keys, int64_t n_build, const void* probe_keys,
                       int64_t n_probe, int key_bytes, int unique_keys)
{
    return pjo_inner_join(build_keys, n_build, probe_keys, n_probe, key_bytes, unique_keys,
                          (int32_t*)0, (int32_t*)0, 0);
}
