// pj_join.cuh -- per-partition shared-memory hash build and probe.
//
// Reference counterparts: hash_join (hash_join_kernels.cuh:24-200), the
// work split of handle_skewed_data (skewed_data_handler.cuh:21-91) and the
// launch of shared_memory_hash_join (partitioned_join.cuh:178-251).
//
// Work items.  Partition p with b build and q probe tuples becomes S_p x K_p
// items: S_p splits the build side so that every piece fits one table (by
// hash bits -- each probe row then visits one table -- or by position, the
// reference's split, when repeated keys defeat hashing), K_p =
// ceil(q / probe_chunk) splits the probe side (the reference has no probe
// split, so one CTA walks a hot partition's whole probe run).  Items are
// numbered partition-major, then probe chunk, then build piece, so CTAs that
// share data run side by side.  A persistent grid claims items through an
// atomic counter (the next claim is issued while the current item runs).
//
// Tables (shared memory).
//   BUCKET (default): the piece's build tuples sorted by bucket = low hash
//     bits, plus an array of bucket ends (16-bit, two per word).  Built by a
//     counting sort: count pass, block scan, place pass.  8 bytes a tuple for
//     4-byte keys, so one CTA holds ~22 K tuples.
//   COMPACT: the same bucket order, but an entry is 4 bytes: 16 bits of the
//     hash above the bucket bits (a fingerprint) and the tuple's 16-bit
//     index in the item's build range.  One CTA holds ~41 K tuples, so large
//     partitions need no split; a fingerprint hit loads the build tuple
//     (from L2: the item read it moments before) to compare the full key
//     and take its row.
//   OPEN: the reference's layout -- open addressing with linear probing,
//     fill <= 0.5 (HASH_TABLE_OCC, hash_join_kernels.cuh:21), slot
//     abs((int)h % T) (:100-101) or a multiply-high of unused hash bits;
//     a CAS on the row word claims a slot, row == -1 marks it empty, so every
//     key value (the reference's -1 sentinel included) joins.
//
// Output.  Probing has no block-wide barrier: each warp numbers a step's
// matches with ballots (all lanes' first tuple's matches, then the second
// tuple's, ...), reserves their positions with one shared atomic on the
// CTA's entry counter and stores them straight from registers, each store
// instruction one contiguous run.  A CTA claims output space from the
// global counter OUT_CHUNK entries at a time, so global atomics are rare
// (the reference's write_back_buffer, hash_join_kernels.cuh:150-199, does
// one per match past its buffer).  Each CTA's last chunk is only partly used; a fix-up pass
// (join_fixup_plan_kernel / join_fixup_move_kernel) moves the entries above
// the true total into those gaps, so the output is dense.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_device.cuh"
#include "pj_types.cuh"

namespace pj {

constexpr uint32_t EMPTY_ROW = 0xffffffffu;
enum : int { TABLE_BUCKET = 0, TABLE_OPEN = 1, TABLE_COMPACT = 2, TABLE_EXACT = 3 };
constexpr int64_t COMPACT_RANGE = 65536;  // build range a COMPACT entry's index can address

__global__ void zero_job_counts_kernel(const JobOut* __restrict__ outs, int32_t n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) *outs[i].count = 0;
}

struct JoinArgs {
    const uint32_t* build_tuples;
    const uint32_t* probe_tuples;
    const int64_t* build_off;   // partition p = [build_off[p*b_items], build_off[(p+1)*b_items])
    const int64_t* probe_off;
    int32_t b_items;
    int32_t p_items;
    int32_t P;
    int32_t digit_bits;         // top hash bits consumed by partition digits (HASH digits), else 0
    const int32_t* split;       // per partition: log2 S_p (hash split) or S_p (position split)
    const int64_t* item_off;    // exclusive scan of items per partition, P+1 entries
    const int32_t* item_part;   // partition of every item
    int64_t max_items;
    uint32_t* queue;            // item counter (zeroed)
    int32_t cap;                // build tuples one table holds (BUCKET) / slots (OPEN)
    int32_t nb_log2;            // BUCKET, COMPACT, EXACT: log2 of the bucket count
    int32_t row_bits;           // EXACT: low bits of an entry holding the build row
    int32_t probe_chunk;        // tuples
    int32_t position_chunk;     // build tuples per position split piece
    int32_t* out_build;         // nullptr: count only
    int32_t* out_probe;
    int64_t capacity;
    unsigned long long* count;  // device int64: chunk reservations, then the match count
    uint32_t* status;
    int64_t* cta_q;             // per CTA: entries produced
    int64_t* cta_last;          // per CTA: base of its last output chunk (-1: none)
    int32_t* over_build;        // reserved positions >= capacity land here
    int32_t* over_probe;
    int64_t over_cap;
    int64_t* seg;               // fix-up segments
    int32_t max_ctas;           // join CTAs the fix-up records have room for
    const unsigned long long* base_count;  // entries written before the join (heavy keys), or nullptr
    const PartRef* parts;       // batches: per partition (else nullptr)
    const JobOut* outs;         // batches: per join
};

// Items per partition (S_p x K_p) and the split of partition p.
// Batches pass `parts` (the partition's segments); single joins nullptr.
__global__ void join_items_kernel(const int64_t* __restrict__ build_off, const int64_t* __restrict__ probe_off,
                                  int32_t b_items, int32_t p_items, int32_t P,
                                  const int32_t* __restrict__ build_tot, const int32_t* __restrict__ probe_tot,
                                  int32_t cap_per_table, int32_t probe_chunk, int32_t hash_split,
                                  int32_t max_split_log2, int32_t* __restrict__ split_out,
                                  int64_t* __restrict__ items_out, uint32_t* __restrict__ status,
                                  const PartRef* __restrict__ parts)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    int64_t b_at = static_cast<int64_t>(p) * b_items, p_at = static_cast<int64_t>(p) * p_items;
    if (parts) {
        b_at = parts[p].b_at;
        p_at = parts[p].p_at;
        b_items = parts[p].b_items;
        p_items = parts[p].p_items;
    }
    const int64_t bc = build_tot[p], pc = probe_tot[p];
    const int64_t prange = probe_off[p_at + p_items] - probe_off[p_at];
    int64_t items = 0;
    int32_t split = 0;
    if (bc > 0 && pc > 0) {
        int64_t S;
        if (hash_split) {
            // hash pieces are only about equal: aim each at 15/16 of a table
            const int64_t target = cap_per_table - cap_per_table / 16;
            int lg = 0;
            while (lg < max_split_log2 && (bc + (1ll << lg) - 1) / (1ll << lg) > target) ++lg;
            split = lg;
            S = 1ll << lg;
        } else {
            const int64_t brange = build_off[b_at + b_items] - build_off[b_at];
            S = (brange + cap_per_table - 1) / cap_per_table;
            if (S < 1) S = 1;
            split = static_cast<int32_t>(S);
        }
        const int64_t K = (prange + probe_chunk - 1) / probe_chunk;
        items = S * K;
    }
    split_out[p] = split;
    items_out[p] = items;
}

// item_part[item_off[p] + k] = p for k < items of p.
__global__ void items_expand_kernel(const int64_t* __restrict__ item_off, int32_t P, int32_t* __restrict__ item_part,
                                    int64_t max_items, uint32_t* __restrict__ status)
{
    const int p = blockIdx.x;
    if (p >= P) return;
    const int64_t a = item_off[p], b = item_off[p + 1];
    if (b > max_items) {
        if (threadIdx.x == 0) raise_status(status, ST_OVERFLOW);
        return;
    }
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) item_part[i] = p;
}

// ---------------------------------------------------------------------------
// L2 residency.  Probe tuples and output entries stream through once; the
// item's build tuples are re-read (place pass, COMPACT verification).  The
// streams are tagged evict-first so that they do not push the build range
// out of L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void st_stream(int32_t* p, int32_t v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}

// Predicated forms: lanes with pred == false skip the access.  One
// predicated instruction each, so the hot loops carry no divergent branch
// around them.
__device__ __forceinline__ void st_stream_if(int32_t* p, int32_t v, bool pred, uint64_t pol)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.L2::cache_hint.b32 [%0], %1, %3;\n\t}"
                 ::"l"(p), "r"(v), "r"(static_cast<uint32_t>(pred)), "l"(pol)
                 : "memory");
}
// v keeps its value where pred is false
__device__ __forceinline__ void ld_stream_if(uint2& v, const uint2* p, bool pred, uint64_t pol)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t"
                 "@q ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %4;\n\t}"
                 : "+r"(v.x), "+r"(v.y)
                 : "l"(p), "r"(static_cast<uint32_t>(pred)), "l"(pol));
}
__device__ __forceinline__ void ld_stream_if(uint4& v, const uint4* p, bool pred, uint64_t pol)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
                 "@q ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %6;\n\t}"
                 : "+r"(v.x), "+r"(v.y), "+r"(v.z), "+r"(v.w)
                 : "l"(p), "r"(static_cast<uint32_t>(pred)), "l"(pol));
}

// ---------------------------------------------------------------------------
// Tuple access: a probe/build tuple gives (hash, comparable key, row).
// 4-byte keys: the stored word 0 is murmur(key), a bijection, so the hash is
// the key.  8-byte keys: the key and its hash are both stored.
template <typename K> struct TupleView;

template <> struct TupleView<int32_t> {
    static constexpr int WORDS = 2;
    using Cmp = uint32_t;
    __device__ __forceinline__ static void load(const uint32_t* base, int64_t i, uint32_t& h, Cmp& key, int32_t& row)
    {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(base) + i);
        h = v.x;
        key = v.x;
        row = static_cast<int32_t>(v.y);
    }
    // row = -1 where pred is false
    __device__ __forceinline__ static void load_stream_if(const uint32_t* base, int64_t i, bool pred, uint32_t& h,
                                                          Cmp& key, int32_t& row, uint64_t pol)
    {
        uint2 v = make_uint2(0u, 0xffffffffu);
        ld_stream_if(v, reinterpret_cast<const uint2*>(base) + i, pred, pol);
        h = v.x;
        key = v.x;
        row = static_cast<int32_t>(v.y);
    }
    __device__ __forceinline__ static void load_key_row(const uint32_t* base, int64_t i, Cmp& key, int32_t& row)
    {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(base) + i);
        key = v.x;
        row = static_cast<int32_t>(v.y);
    }
};

template <> struct TupleView<int64_t> {
    static constexpr int WORDS = 4;  // {key_lo, key_hi, hash, row}
    using Cmp = unsigned long long;
    __device__ __forceinline__ static void load(const uint32_t* base, int64_t i, uint32_t& h, Cmp& key, int32_t& row)
    {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(base) + i);
        key = (static_cast<unsigned long long>(v.y) << 32) | v.x;
        h = v.z;
        row = static_cast<int32_t>(v.w);
    }
    __device__ __forceinline__ static void load_stream_if(const uint32_t* base, int64_t i, bool pred, uint32_t& h,
                                                          Cmp& key, int32_t& row, uint64_t pol)
    {
        uint4 v = make_uint4(0u, 0u, 0u, 0xffffffffu);
        ld_stream_if(v, reinterpret_cast<const uint4*>(base) + i, pred, pol);
        key = (static_cast<unsigned long long>(v.y) << 32) | v.x;
        h = v.z;
        row = static_cast<int32_t>(v.w);
    }
    __device__ __forceinline__ static void load_key_row(const uint32_t* base, int64_t i, Cmp& key, int32_t& row)
    {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(base) + i);
        key = (static_cast<unsigned long long>(v.y) << 32) | v.x;
        row = static_cast<int32_t>(v.w);
    }
};

// Entry of an EXACT table: the tag (hash bits above the bucket bits) << R |
// build row, R = row bits.  A 4-byte key is its MurmurHash3 value (a
// bijection), so the tag, the bucket and the partition's hash digits fix the
// key.  For an 8-byte key MurmurHash3_x86_32 maps the high word to the hash
// bijectively for each low word (the second block's mixing, rotation,
// multiply-add, length xor and fmix32 are all invertible), so (low word,
// hash) fixes the key: the entry keeps the low word beside the tag.
template <typename K> struct ExactEntry;
template <> struct ExactEntry<int32_t> {
    static constexpr int BYTES = 4;
    __device__ __forceinline__ static void put(uint8_t* t, int i, uint32_t tag, uint32_t) { reinterpret_cast<uint32_t*>(t)[i] = tag; }
    __device__ __forceinline__ static uint32_t get(const uint8_t* t, int i, uint32_t& key_lo)
    {
        key_lo = 0u;
        return reinterpret_cast<const uint32_t*>(t)[i];
    }
    __device__ __forceinline__ static uint32_t key_lo(uint32_t) { return 0u; }
};
template <> struct ExactEntry<int64_t> {
    static constexpr int BYTES = 8;
    __device__ __forceinline__ static void put(uint8_t* t, int i, uint32_t tag, uint32_t lo)
    {
        reinterpret_cast<uint2*>(t)[i] = make_uint2(lo, tag);
    }
    __device__ __forceinline__ static uint32_t get(const uint8_t* t, int i, uint32_t& key_lo)
    {
        const uint2 v = reinterpret_cast<const uint2*>(t)[i];
        key_lo = v.x;
        return v.y;
    }
    __device__ __forceinline__ static uint32_t key_lo(unsigned long long k) { return static_cast<uint32_t>(k); }
};

// One pass of the predicated bucket walk for one probe tuple, in PTX so that
// the cursor test, the skipped load and the updates are all predicated
// instructions.  at / end: shared-window byte addresses of the tuple's
// cursor and of its bucket's end; a lane whose cursor has reached the end
// skips the load (no wavefront, no bank conflict).  A match sets end = at,
// so the walk stops with at = end + the entry size: afterwards at > end
// marks a match, whose row word is the 4 bytes below at (walk_row).
//
// 4-byte EXACT entries: e matches when (e ^ fqs) < lim, i.e. its bits above
// the row bits equal the tuple's tag (fqs = tag << R, lim = 1 << R).
__device__ __forceinline__ void walk_exact4(uint32_t& at, uint32_t& end, uint32_t fqs, uint32_t lim)
{
    asm volatile("{\n\t.reg .pred p, q;\n\t.reg .b32 e, t;\n\t"
                 "setp.lt.u32 p, %0, %1;\n\t"
                 "@p ld.shared.u32 e, [%0];\n\t"
                 "xor.b32 t, e, %2;\n\t"
                 "setp.lt.and.u32 q, t, %3, p;\n\t"
                 "@q mov.b32 %1, %0;\n\t"
                 "@p add.u32 %0, %0, 4;\n\t"
                 "}"
                 : "+r"(at), "+r"(end)
                 : "r"(fqs), "r"(lim));
}

// 8-byte EXACT entries {key low word, tag << R | row}: the low word must
// equal the tuple's too.
__device__ __forceinline__ void walk_exact8(uint32_t& at, uint32_t& end, uint32_t fqs, uint32_t lim, uint32_t klo)
{
    asm volatile("{\n\t.reg .pred p, q;\n\t.reg .b32 lo, e, t;\n\t"
                 "setp.lt.u32 p, %0, %1;\n\t"
                 "@p ld.shared.v2.u32 {lo, e}, [%0];\n\t"
                 "xor.b32 t, e, %2;\n\t"
                 "setp.lt.and.u32 q, t, %3, p;\n\t"
                 "setp.eq.and.u32 q, lo, %4, q;\n\t"
                 "@q mov.b32 %1, %0;\n\t"
                 "@p add.u32 %0, %0, 8;\n\t"
                 "}"
                 : "+r"(at), "+r"(end)
                 : "r"(fqs), "r"(lim), "r"(klo));
}

// 8-byte BUCKET entries {key, row} of 4-byte keys: a match is key == k.
__device__ __forceinline__ void walk_bucket8(uint32_t& at, uint32_t& end, uint32_t k)
{
    asm volatile("{\n\t.reg .pred p, q;\n\t.reg .b32 ek;\n\t"
                 "setp.lt.u32 p, %0, %1;\n\t"
                 "@p ld.shared.u32 ek, [%0];\n\t"
                 "setp.eq.and.u32 q, ek, %2, p;\n\t"
                 "@q mov.b32 %1, %0;\n\t"
                 "@p add.u32 %0, %0, 8;\n\t"
                 "}"
                 : "+r"(at), "+r"(end)
                 : "r"(k));
}

// After a walk: whether the cursor stopped on a match, and that entry's row
// word (its last 4 bytes, just below the cursor); 0 without a match.
__device__ __forceinline__ uint32_t walk_row(uint32_t at, uint32_t end)
{
    uint32_t v = 0u;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.gt.u32 p, %1, %2;\n\t@p ld.shared.u32 %0, [%3];\n\t}"
                 : "+r"(v)
                 : "r"(at), "r"(end), "r"(at - 4u));
    return v;
}

// Entry of a BUCKET table.
template <typename K> struct Entry;
template <> struct Entry<int32_t> {
    static constexpr int BYTES = 8;  // {hash/key, row}
    __device__ __forceinline__ static void put(uint8_t* t, int i, uint32_t key, int32_t row)
    {
        reinterpret_cast<uint2*>(t)[i] = make_uint2(key, static_cast<uint32_t>(row));
    }
    __device__ __forceinline__ static void get(const uint8_t* t, int i, uint32_t& key, uint32_t& row)
    {
        const uint2 v = reinterpret_cast<const uint2*>(t)[i];
        key = v.x;
        row = v.y;
    }
};
template <> struct Entry<int64_t> {
    static constexpr int BYTES = 12;  // {lo, hi, row}
    __device__ __forceinline__ static void put(uint8_t* t, int i, unsigned long long key, int32_t row)
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(t) + 3 * i;
        w[0] = static_cast<uint32_t>(key);
        w[1] = static_cast<uint32_t>(key >> 32);
        w[2] = static_cast<uint32_t>(row);
    }
    __device__ __forceinline__ static void get(const uint8_t* t, int i, unsigned long long& key, uint32_t& row)
    {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(t) + 3 * i;
        key = (static_cast<unsigned long long>(w[1]) << 32) | w[0];
        row = w[2];
    }
};

// Asynchronous prefetch of a byte range into L2 (the bulk-copy engine's
// prefetch form): 16-byte aligned start, issued in 64 KB pieces.
__device__ __forceinline__ void prefetch_l2(const void* p, int64_t bytes)
{
    const uint8_t* c = static_cast<const uint8_t*>(p);
    for (int64_t off = 0; off < bytes; off += 65536) {
        const int64_t left = bytes - off;
        const uint32_t n = static_cast<uint32_t>((left < 65536 ? left : 65536) & ~int64_t(15));
        if (n) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + off), "r"(n) : "memory");
    }
}

// The same for data read once (probe chunks): tagged evict-first.
__device__ __forceinline__ void prefetch_l2_stream(const void* p, int64_t bytes, uint64_t pol)
{
    const uint8_t* c = static_cast<const uint8_t*>(p);
    for (int64_t off = 0; off < bytes; off += 65536) {
        const int64_t left = bytes - off;
        const uint32_t n = static_cast<uint32_t>((left < 65536 ? left : 65536) & ~int64_t(15));
        if (n)
            asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(c + off), "r"(n),
                         "l"(pol)
                         : "memory");
    }
}

// Bytes of a probe chunk prefetched into L2 at an item's start.  The whole
// chunk (~1 MB, 148 CTAs at once: more than L2 holds) was evicted before the
// warps reached its tail and read twice; a 128 KB head measured best (2^26 x
// 2^28 int64 join 7.42 -> 6.62 ms, 2^27 x 2^27 int32 2.47 -> 2.44 ms).
constexpr int64_t PROBE_PREFETCH_BYTES = 128 << 10;

// Output geometry.
constexpr int OUT_CHUNK = 8192;  // entries a CTA claims per global atomic
constexpr int OUT_SLOTS = 16;    // chunk bases a CTA keeps in shared memory
constexpr int JOIN_U = 4;        // probe tuples in flight per lane
constexpr int JOIN_BU = 4;       // build tuples in flight per thread

// Where one work item's tuples are.  Thread 0 works it out for the next
// item while the current one probes, so an item starts without a chain of
// dependent global loads (item -> partition -> offsets).
struct ItemMeta {
    int64_t b_lo, b_hi;  // build tuples of the item's piece
    int64_t q_lo, q_hi;  // probe tuples of the item's chunk
    int32_t p;           // partition
    int32_t piece;       // build piece (hash split: the piece's hash bits)
    int32_t sbits;       // hash split bits (0: no hash split)
    int32_t dbits;       // top hash bits the partition digits consumed
    JobOut jout;         // batches: the item's join
};

template <typename K, int TABLE>
struct JoinSmem {
    // table bytes for capacity cap (BUCKET: tuples; OPEN: slots) and 2^nb_log2 buckets
    __host__ __device__ static size_t entries_bytes(int cap)
    {
        const size_t e = TABLE == TABLE_OPEN                                    ? (sizeof(K) == 4 ? 8 : 12)
                         : TABLE == TABLE_EXACT                                ? ExactEntry<K>::BYTES
                         : TABLE == TABLE_COMPACT                              ? 4
                                                                            : Entry<K>::BYTES;
        return (static_cast<size_t>(cap) * e + 127) & ~size_t(127);
    }
    __host__ __device__ static size_t table_bytes(int cap, int nb_log2)
    {
        size_t t = entries_bytes(cap);
        if (TABLE != TABLE_OPEN) t += ((static_cast<size_t>(1) << nb_log2) / 2 + 1) * 4;
        return (t + 127) & ~size_t(127);
    }
    // dynamic shared memory of a join CTA: the table alone (matches go
    // straight from registers to global memory)
    __host__ __device__ static size_t bytes(int cap, int nb_log2) { return table_bytes(cap, nb_log2); }
};

template <typename K, int TABLE, bool UNIQUE, bool HASH_SPLIT, bool SLOT_REF, int THREADS, bool BATCH = false>
__global__ void __launch_bounds__(THREADS, 1) join_kernel(JoinArgs a)
{
    using TV = TupleView<K>;
    using Cmp = typename TV::Cmp;
    using E = Entry<K>;
    using SM = JoinSmem<K, TABLE>;
    constexpr int NWARPS = THREADS / 32;
    const int lane = threadIdx.x & 31;
    constexpr int U = JOIN_U;

    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* table = smem;
    uint32_t* ends = reinterpret_cast<uint32_t*>(smem + SM::entries_bytes(a.cap));
    // OPEN tables of 8-byte keys: keys[cap] (8 B) then rows[cap]
    unsigned long long* okeys = reinterpret_cast<unsigned long long*>(table);
    uint32_t* ctab = reinterpret_cast<uint32_t*>(table);  // COMPACT: fingerprint << 16 | index
    uint32_t* orows = reinterpret_cast<uint32_t*>(table + static_cast<size_t>(a.cap) * 8);

    __shared__ int64_t s_item, s_next;
    __shared__ uint32_t s_q;                  // entries this CTA produced
    __shared__ unsigned long long s_cslot[OUT_SLOTS];  // (chunk << 40) | base, ~0: empty
    __shared__ uint32_t s_warp[NWARPS];
    __shared__ int s_nbuild;
    __shared__ uint32_t s_step;  // next probe step of the current item
    __shared__ ItemMeta s_cur, s_nxt;  // the current and the next item

    const uint64_t stream_pol = l2_evict_first_policy();
    const int NB = 1 << a.nb_log2;
    const uint32_t nb_mask = static_cast<uint32_t>(NB - 1);
    const int64_t total_items = a.item_off[a.P];
    const bool write_out = a.out_build != nullptr;

    auto load_meta = [&](int64_t it) -> ItemMeta {
        ItemMeta m;
        const int p = a.item_part[it];
        const int64_t local = it - a.item_off[p];
        const int32_t split = a.split[p];
        const int64_t S = HASH_SPLIT ? (1ll << split) : split;
        const int64_t piece = local % S;
        const int64_t pchunk = local / S;
        int64_t b_at = static_cast<int64_t>(p) * a.b_items, p_at = static_cast<int64_t>(p) * a.p_items;
        int32_t b_n = a.b_items, p_n = a.p_items;
        m.dbits = a.digit_bits;
        m.jout = JobOut{};
        if constexpr (BATCH) {
            const PartRef r = a.parts[p];
            b_at = r.b_at;
            p_at = r.p_at;
            b_n = r.b_items;
            p_n = r.p_items;
            m.dbits = r.digit_bits;
            m.jout = a.outs[r.job];
        }
        const int64_t b_lo0 = a.build_off[b_at];
        const int64_t b_hi0 = a.build_off[b_at + b_n];
        m.b_lo = b_lo0;
        m.b_hi = b_hi0;
        if (!HASH_SPLIT) {
            m.b_lo = b_lo0 + piece * a.position_chunk;
            m.b_hi = m.b_lo + a.position_chunk < b_hi0 ? m.b_lo + a.position_chunk : b_hi0;
            if (m.b_lo > m.b_hi) m.b_lo = m.b_hi;
        }
        const int64_t q_lo0 = a.probe_off[p_at];
        const int64_t q_hi0 = a.probe_off[p_at + p_n];
        m.q_lo = q_lo0 + pchunk * a.probe_chunk;
        m.q_hi = m.q_lo + a.probe_chunk < q_hi0 ? m.q_lo + a.probe_chunk : q_hi0;
        m.p = p;
        m.piece = static_cast<int32_t>(piece);
        m.sbits = HASH_SPLIT ? split : 0;
        return m;
    };
    if (threadIdx.x == 0) {
        s_q = 0;
        s_next = static_cast<int64_t>(atomicAdd(a.queue, 1u));
        if (s_next < total_items && s_next < a.max_items) s_nxt = load_meta(s_next);
    }
    if (threadIdx.x < OUT_SLOTS) s_cslot[threadIdx.x] = ~0ull;

    // -- output ------------------------------------------------------------
    // Base of output chunk ch: reserved with one global atomic by the lane
    // whose entries include the chunk's first position, read by the others.
    // A slot holds (ch << 40) | base in one 64-bit word, so a reader sees a
    // consistent pair without a memory fence (a fence would wait for the
    // thread's outstanding global stores).
    auto chunk_base = [&](uint32_t ch, bool reserve) -> long long {
        const int slot = static_cast<int>(ch % OUT_SLOTS);
        volatile unsigned long long* vslot = s_cslot;
        if (reserve) {
            const unsigned long long g = atomicAdd(a.count, static_cast<unsigned long long>(OUT_CHUNK));
            vslot[slot] = (static_cast<unsigned long long>(ch) << 40) | g;
            return static_cast<long long>(g);
        }
        uint32_t spins = 0;
        for (;;) {
            const unsigned long long v = vslot[slot];
            if (v != ~0ull) {
                const uint32_t c = static_cast<uint32_t>(v >> 40);
                if (c == ch) return static_cast<long long>(v & ((1ull << 40) - 1));
                if (c > ch) {  // slot reused: cannot happen with OUT_SLOTS of slack
                    raise_status(a.status, ST_INTERNAL);
                    return -1;
                }
            }
            if (++spins > SPIN_LIMIT) {
                raise_status(a.status, ST_TIMEOUT);
                return -1;
            }
            __nanosleep(20);
        }
    };
    auto store_out = [&](long long pos, int32_t b, int32_t q) {
        if (pos < a.capacity) {
            a.out_build[pos] = b;
            a.out_probe[pos] = q;
        } else if (pos - a.capacity < a.over_cap) {
            a.over_build[pos - a.capacity] = b;
            a.over_probe[pos - a.capacity] = q;
        } else {
            raise_status(a.status, ST_CAPACITY);
        }
    };
    JobOut jout{};  // batches: the current item's join
    // Whole warp: lane l appends (brow[u], rp[u]) for every u with emit[u].
    // The step's entries are laid out u-major (all lanes' u = 0 entries, then
    // u = 1, ...), so each store instruction writes one contiguous run and
    // no staging buffer is needed.
    auto append_direct = [&](const bool (&emit)[U], const uint32_t (&brow)[U], const int32_t (&rp)[U]) {
        const uint32_t lt = (1u << lane) - 1u;
        int off[U];
        int n = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t m = __ballot_sync(0xffffffffu, emit[u]);
            off[u] = n + __popc(m & lt);
            n += __popc(m);
        }
        if (n == 0) return;
        if constexpr (BATCH) {
            // exact positions in the join's own output: one atomic per warp step
            unsigned long long q0 = 0;
            if (lane == 0) q0 = atomicAdd(jout.count, static_cast<unsigned long long>(n));
            q0 = __shfl_sync(0xffffffffu, q0, 0);
            if (jout.out_build == nullptr) return;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (emit[u]) {
                    const long long pos = static_cast<long long>(q0) + off[u];
                    if (pos < jout.capacity) {
                        st_stream(jout.out_build + pos, static_cast<int32_t>(brow[u]), stream_pol);
                        st_stream(jout.out_probe + pos, rp[u], stream_pol);
                    } else {
                        raise_status(a.status, ST_CAPACITY);
                    }
                }
            return;
        }
        uint32_t q0 = 0;
        if (lane == 0) q0 = atomicAdd(&s_q, static_cast<uint32_t>(n));
        q0 = __shfl_sync(0xffffffffu, q0, 0);
        if (!write_out) return;  // count only
        const uint32_t ch0 = q0 / OUT_CHUNK, ch1 = (q0 + n - 1) / OUT_CHUNK;
        const bool first = q0 % OUT_CHUNK == 0;
        if (first || ch1 != ch0) {  // rare: the step holds a chunk's first position and reserves it
            if (lane == 0 && first) chunk_base(ch0, true);
            if (lane == 1 && ch1 != ch0) chunk_base(ch1, true);
            __syncwarp();
        }
        // every lane reads the bases (one broadcast load): no divergent lane
        const long long b0 = chunk_base(ch0, false);
        const long long b1 = ch1 != ch0 ? chunk_base(ch1, false) : 0;
        // entries [0, n0) go to chunk ch0 from position p0, the rest to ch1
        const int n0 = ch1 == ch0 ? n : static_cast<int>(ch1 * OUT_CHUNK - q0);
        const long long p0 = b0 + static_cast<long long>(q0 % OUT_CHUNK);
        const long long p1 = b1 - n0;
        if (n0 == n && b0 >= 0 && p0 + n <= a.capacity) {  // one chunk: the common case
            int32_t* ob = a.out_build + p0;
            int32_t* op = a.out_probe + p0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                st_stream_if(ob + off[u], static_cast<int32_t>(brow[u]), emit[u], stream_pol);
                st_stream_if(op + off[u], rp[u], emit[u], stream_pol);
            }
        } else if (b0 >= 0 && p0 + n0 <= a.capacity && (n0 == n || (b1 >= 0 && b1 + (n - n0) <= a.capacity))) {
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (emit[u]) {
                    const long long pos = (off[u] < n0 ? p0 : p1) + off[u];
                    st_stream(a.out_build + pos, static_cast<int32_t>(brow[u]), stream_pol);
                    st_stream(a.out_probe + pos, rp[u], stream_pol);
                }
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (emit[u]) {
                    if (off[u] < n0) {
                        if (b0 >= 0) store_out(p0 + off[u], static_cast<int32_t>(brow[u]), rp[u]);
                    } else if (b1 >= 0) {
                        store_out(p1 + off[u], static_cast<int32_t>(brow[u]), rp[u]);
                    }
                }
        }
    };
    bool first_item = true;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_item = s_next;
            s_cur = s_nxt;
            s_next = static_cast<int64_t>(atomicAdd(a.queue, 1u));  // claim the next item early
        }
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total_items || item >= a.max_items) break;
        const int p = s_cur.p;
        const int64_t piece = s_cur.piece;
        const int sbits = s_cur.sbits;
        const int dbits = s_cur.dbits;
        const int64_t b_lo = s_cur.b_lo, b_hi = s_cur.b_hi;
        const int64_t q_lo = s_cur.q_lo, q_hi = s_cur.q_hi;
        if constexpr (BATCH) jout = s_cur.jout;
        const int skip = dbits + sbits;
        const int piece_shift = 32 - (sbits > 0 ? sbits : 1);

        // a CTA's first item: its build range was not prefetched during an
        // earlier probe phase
        if (TABLE != TABLE_COMPACT && first_item && threadIdx.x == 0 && b_hi > b_lo) {
            const int64_t bbytes = (b_hi - b_lo) * TV::WORDS * 4;
            prefetch_l2(a.build_tuples + b_lo * TV::WORDS, bbytes < (1 << 20) ? bbytes : (1 << 20));
        }
        first_item = false;
        // the head of the probe chunk streams into L2 while the table is built
        if (threadIdx.x == 0) {
            const int64_t pbytes = (q_hi - q_lo) * TV::WORDS * 4;
            prefetch_l2_stream(a.probe_tuples + (q_lo * TV::WORDS),
                               pbytes < PROBE_PREFETCH_BYTES ? pbytes : PROBE_PREFETCH_BYTES, stream_pol);
        }

        auto in_piece = [&](uint32_t h) -> bool {
            if (!HASH_SPLIT || sbits == 0) return true;
            return static_cast<int64_t>((h << dbits) >> piece_shift) == piece;
        };
        auto bucket_of = [&](uint32_t h) -> uint32_t { return h & nb_mask; };
        auto finger_of = [&](uint32_t h) -> uint32_t { return (h >> a.nb_log2) & 0xffffu; };
        // EXACT entries: (hash bits above the bucket bits) << row_bits | build row;
        // with the digits' and the bucket's bits they fix the whole hash
        const uint32_t x_rmask = (1u << a.row_bits) - 1u;
        auto xfinger_of = [&](uint32_t h) -> uint32_t { return (h >> a.nb_log2) & (0xffffffffu >> a.row_bits); };
        auto slot_of = [&](uint32_t h) -> uint32_t {
            return SLOT_REF ? slot_ref(h, a.cap) : slot_fast(h, skip, static_cast<uint32_t>(a.cap));
        };

        if (threadIdx.x == 0) s_step = 0;  // ordered before the probe by the build's barriers

        // ---- build ----
        bool skip_item = false;
        if (TABLE == TABLE_COMPACT && b_hi - b_lo > COMPACT_RANGE) {
            // an entry's 16-bit index cannot address this range: the planner avoids it
            if (threadIdx.x == 0) raise_status(a.status, ST_OVERFLOW);
            skip_item = true;
            __syncthreads();
        } else if constexpr (TABLE != TABLE_OPEN) {
            // bucket directory: 16-bit counts of bucket b at index b + 1; after
            // the scan and the place pass index b holds the start of bucket b
            // and index b + 1 its end
            for (int i = threadIdx.x; i <= NB / 2; i += THREADS) ends[i] = 0u;
            if (threadIdx.x == 0) s_nbuild = 0;
            __syncthreads();
            // pass 1: count per bucket; the next batch of loads is issued
            // before the current one is counted
            int mine = 0;
            {
                uint32_t nh[JOIN_BU];
                Cmp nk[JOIN_BU];
                int32_t nr[JOIN_BU];
                // 32-bit offsets in the item's build range
                const uint32_t* bt = a.build_tuples + b_lo * TV::WORDS;
                const uint32_t bn = static_cast<uint32_t>(b_hi - b_lo);
                auto load_batch = [&](uint32_t i0) {
#pragma unroll
                    for (int u = 0; u < JOIN_BU; ++u) {
                        const uint32_t i = i0 + u * THREADS;
                        nr[u] = -1;
                        if (i < bn) TV::load(bt, i, nh[u], nk[u], nr[u]);
                    }
                };
                uint32_t i0 = threadIdx.x;
                if (i0 < bn) load_batch(i0);
                for (; i0 < bn; i0 += THREADS * JOIN_BU) {
                    uint32_t h[JOIN_BU];
                    int32_t r[JOIN_BU];
#pragma unroll
                    for (int u = 0; u < JOIN_BU; ++u) {
                        h[u] = nh[u];
                        r[u] = nr[u];
                    }
                    if (i0 + THREADS * JOIN_BU < bn) load_batch(i0 + THREADS * JOIN_BU);
#pragma unroll
                    for (int u = 0; u < JOIN_BU; ++u) {
                        if (r[u] >= 0 && in_piece(h[u])) {
                            const uint32_t b = bucket_of(h[u]) + 1u;
                            atomicAdd(&ends[b >> 1], (b & 1u) ? 0x10000u : 1u);
                            ++mine;
                        }
                    }
                }
            }
            mine = __reduce_add_sync(0xffffffffu, mine);
            if (lane == 0 && mine) atomicAdd(&s_nbuild, mine);
            __syncthreads();
            if (s_nbuild > a.cap) {  // the planner sizes pieces to fit; flag and skip
                if (threadIdx.x == 0) raise_status(a.status, ST_OVERFLOW);
                skip_item = true;
            } else {
                scan_u16_pairs<THREADS>(ends, NB / 2 + 1, s_warp);
                // pass 2: place
                const uint32_t* bt = a.build_tuples + b_lo * TV::WORDS;
                const uint32_t bn = static_cast<uint32_t>(b_hi - b_lo);
                for (uint32_t i0 = threadIdx.x; i0 < bn; i0 += THREADS * JOIN_BU) {
                    uint32_t h[JOIN_BU];
                    Cmp k[JOIN_BU];
                    int32_t r[JOIN_BU];
#pragma unroll
                    for (int u = 0; u < JOIN_BU; ++u) {
                        const uint32_t i = i0 + u * THREADS;
                        r[u] = -1;
                        if (i < bn) TV::load(bt, i, h[u], k[u], r[u]);
                    }
#pragma unroll
                    for (int u = 0; u < JOIN_BU; ++u) {
                        if (r[u] >= 0 && in_piece(h[u])) {
                            const uint32_t b = bucket_of(h[u]) + 1u;
                            const uint32_t old = atomicAdd(&ends[b >> 1], (b & 1u) ? 0x10000u : 1u);
                            const int pos = static_cast<int>((b & 1u) ? (old >> 16) : (old & 0xffffu));
                            if constexpr (TABLE == TABLE_COMPACT)
                                ctab[pos] = (finger_of(h[u]) << 16) | (i0 + u * THREADS);
                            else if constexpr (TABLE == TABLE_EXACT)
                                ExactEntry<K>::put(table, pos, (xfinger_of(h[u]) << a.row_bits) | static_cast<uint32_t>(r[u]),
                                                   ExactEntry<K>::key_lo(k[u]));
                            else
                                E::put(table, pos, k[u], r[u]);
                        }
                    }
                }
            }
            __syncthreads();
        } else {
            for (int i = threadIdx.x; i < a.cap; i += THREADS) {
                if constexpr (sizeof(K) == 4) reinterpret_cast<uint2*>(table)[i] = make_uint2(0u, EMPTY_ROW);
                else orows[i] = EMPTY_ROW;
            }
            __syncthreads();
            for (int64_t i = b_lo + threadIdx.x; i < b_hi; i += THREADS) {
                uint32_t h;
                Cmp k;
                int32_t r;
                TV::load(a.build_tuples, i, h, k, r);
                if (r < 0 || !in_piece(h)) continue;
                uint32_t sl = slot_of(h);
                int tries = 0;
                for (;;) {
                    uint32_t* rw = sizeof(K) == 4 ? &reinterpret_cast<uint2*>(table)[sl].y : &orows[sl];
                    if (atomicCAS(rw, EMPTY_ROW, static_cast<uint32_t>(r)) == EMPTY_ROW) {
                        if constexpr (sizeof(K) == 4) reinterpret_cast<uint2*>(table)[sl].x = static_cast<uint32_t>(k);
                        else okeys[sl] = k;
                        break;
                    }
                    if (++sl == static_cast<uint32_t>(a.cap)) sl = 0;
                    if (++tries >= a.cap) {
                        raise_status(a.status, ST_OVERFLOW);
                        break;
                    }
                }
            }
            __syncthreads();
        }

        // the next item's build side streams into L2 while this item probes,
        // so the next build's count pass reads L2 (BUCKET tables: 8% at
        // 2^25; EXACT tables: 2^27 x 2^27 int32 join 1.72 -> 1.59 ms).  Not
        // for COMPACT tables: their fingerprint checks re-read build tuples
        // and the prefetched ranges were evicted before use (0.83 GB more
        // DRAM reads at 2^27 x 2^27, no time gained).
        if (threadIdx.x == 0 && s_next < total_items && s_next < a.max_items) {
            s_nxt = load_meta(s_next);
            if (TABLE != TABLE_COMPACT && s_nxt.p != p && s_nxt.b_hi > s_nxt.b_lo) {
                const int64_t nbytes = (s_nxt.b_hi - s_nxt.b_lo) * TV::WORDS * 4;
                prefetch_l2(a.build_tuples + s_nxt.b_lo * TV::WORDS, nbytes < (1 << 20) ? nbytes : (1 << 20));
            }
        }

        // ---- probe: warps run independently; loads run one step ahead ----
        if (!skip_item) {
            // warps claim steps of 32*U tuples from a shared counter, so they
            // finish the item together; the next claim's loads run ahead
            const uint32_t* pbase = a.probe_tuples + q_lo * TV::WORDS;
            const uint32_t qn = static_cast<uint32_t>(q_hi - q_lo);
            constexpr uint32_t STEP = 32 * U;
            uint32_t nh[U];
            Cmp nk[U];
            int32_t nr[U];
            auto claim = [&]() -> uint32_t {
                uint32_t st = 0;
                if (lane == 0) st = atomicAdd(&s_step, 1u);
                return __shfl_sync(0xffffffffu, st, 0) * STEP;
            };
            auto load_step = [&](uint32_t s0) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t i = s0 + u * 32 + lane;
                    TV::load_stream_if(pbase, i, i < qn, nh[u], nk[u], nr[u], stream_pol);
                }
            };
            uint32_t s0 = claim();
            if (s0 < qn) load_step(s0);
            while (s0 < qn) {
                uint32_t h[U];
                Cmp k[U];
                int32_t r[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    h[u] = nh[u];
                    k[u] = nk[u];
                    r[u] = nr[u];
                }
                const uint32_t s_after = claim();
                if (s_after < qn) load_step(s_after);
                // look up one tuple from (at, end) or slot sl; returns whether a match was found
                auto lookup = [&](int u, int& at_u, int end_u, uint32_t& sl_u, int& steps_u, bool& live_u,
                                  uint32_t& brow_u) -> bool {
                    bool found = false;
                    if constexpr (TABLE == TABLE_COMPACT) {
                        const uint32_t fq = finger_of(h[u]);
                        while (at_u < end_u) {
                            const uint32_t e = ctab[at_u];
                            ++at_u;
                            if ((e >> 16) == fq) {  // fingerprint hit: compare the full key
                                Cmp bk;
                                int32_t br;
                                TV::load_key_row(a.build_tuples, b_lo + (e & 0xffffu), bk, br);
                                if (bk == k[u]) {
                                    found = true;
                                    brow_u = static_cast<uint32_t>(br);
                                    break;
                                }
                            }
                        }
                        if (!found || UNIQUE) live_u = false;
                    } else if constexpr (TABLE == TABLE_EXACT) {
                        const uint32_t fq = xfinger_of(h[u]), klo = ExactEntry<K>::key_lo(k[u]);
                        while (at_u < end_u) {
                            uint32_t elo;
                            const uint32_t e = ExactEntry<K>::get(table, at_u, elo);
                            ++at_u;
                            if ((e >> a.row_bits) == fq && elo == klo) {  // the key is equal
                                found = true;
                                brow_u = e & x_rmask;
                                break;
                            }
                        }
                        if (!found || UNIQUE) live_u = false;
                    } else if constexpr (TABLE == TABLE_BUCKET) {
                        while (at_u < end_u) {
                            Cmp ek;
                            uint32_t er;
                            E::get(table, at_u, ek, er);
                            ++at_u;
                            if (ek == k[u]) {
                                found = true;
                                brow_u = er;
                                break;
                            }
                        }
                        if (!found || UNIQUE) live_u = false;
                    } else {
                        for (;;) {
                            Cmp ek;
                            uint32_t er;
                            if constexpr (sizeof(K) == 4) {
                                const uint2 v = reinterpret_cast<const uint2*>(table)[sl_u];
                                ek = v.x;
                                er = v.y;
                            } else {
                                er = orows[sl_u];
                                ek = okeys[sl_u];
                            }
                            if (er == EMPTY_ROW) { live_u = false; break; }
                            if (++sl_u == static_cast<uint32_t>(a.cap)) sl_u = 0;
                            if (++steps_u > a.cap) { live_u = false; break; }
                            if (ek == k[u]) {
                                found = true;
                                brow_u = er;
                                if (UNIQUE) live_u = false;
                                break;
                            }
                        }
                    }
                    return found;
                };
                auto start = [&](int u, int& at_u, int& end_u, uint32_t& sl_u) {
                    if constexpr (TABLE != TABLE_OPEN) {
                        const uint16_t* e16 = reinterpret_cast<const uint16_t*>(ends);
                        const uint32_t b = bucket_of(h[u]);
                        at_u = e16[b];
                        end_u = e16[b + 1];
                    } else {
                        sl_u = slot_of(h[u]);
                    }
                };
                if constexpr (UNIQUE && TABLE == TABLE_COMPACT) {
                    // every tuple matches at most once.  The U tuples walk their
                    // buckets in lockstep comparing fingerprints; hits load their
                    // build tuples together; a false hit (equal fingerprint, other
                    // key) resumes its walk.
                    bool emit[U], live[U];
                    uint32_t brow[U], fq[U];
                    int at[U], end[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        emit[u] = false;
                        brow[u] = 0;
                        fq[u] = finger_of(h[u]);
                        live[u] = r[u] >= 0 && in_piece(h[u]);
                        at[u] = end[u] = 0;
                        if (live[u]) {
                            const uint16_t* e16 = reinterpret_cast<const uint16_t*>(ends);
                            const uint32_t b = bucket_of(h[u]);
                            at[u] = e16[b];
                            end[u] = e16[b + 1];
                            live[u] = at[u] < end[u];
                        }
                    }
                    for (;;) {
                        bool hit[U];
#pragma unroll
                        for (int u = 0; u < U; ++u) hit[u] = false;
                        for (;;) {
                            bool any = false;
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                if (live[u]) {
                                    if ((ctab[at[u]] >> 16) == fq[u]) {
                                        hit[u] = true;
                                        live[u] = false;
                                    } else {
                                        live[u] = ++at[u] < end[u];
                                    }
                                }
                                any |= live[u];
                            }
                            if (!any) break;
                        }
                        bool again = false;
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            if (hit[u]) {
                                Cmp bk;
                                int32_t br;
                                TV::load_key_row(a.build_tuples, b_lo + (ctab[at[u]] & 0xffffu), bk, br);
                                if (bk == k[u]) {
                                    emit[u] = true;
                                    brow[u] = static_cast<uint32_t>(br);
                                } else {
                                    live[u] = ++at[u] < end[u];
                                    again |= live[u];
                                }
                            }
                        }
                        if (!__any_sync(0xffffffffu, again)) break;
                    }
                    append_direct(emit, brow, r);
                } else if constexpr (UNIQUE && TABLE == TABLE_EXACT) {
                    // every tuple matches at most once, and an entry's bits decide
                    // it.  Predicated walk: each pass looks at one entry of every
                    // unfinished tuple (walk_exact4/8) and the loop runs while any
                    // lane has one left; finished cursors skip their load.  2^27 x
                    // 2^27 int32 join: 1.72 ms with a branchy lockstep walk, 1.53
                    // with selects, 1.31 with skipped loads and build prefetches.
                    constexpr uint32_t EB = ExactEntry<K>::BYTES;
                    const uint32_t tb = static_cast<uint32_t>(__cvta_generic_to_shared(table));
                    const uint32_t lim = 1u << a.row_bits;
                    bool emit[U];
                    uint32_t brow[U], fqs[U], at[U], end[U];
                    const uint16_t* e16 = reinterpret_cast<const uint16_t*>(ends);
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        fqs[u] = (h[u] >> a.nb_log2) << a.row_bits;  // xfinger_of(h) << R
                        const bool ok = r[u] >= 0 && in_piece(h[u]);
                        const uint32_t b = bucket_of(h[u]);
                        const uint32_t e_lo = e16[b], e_hi = e16[b + 1];
                        at[u] = tb + e_lo * EB;
                        end[u] = ok ? tb + e_hi * EB : at[u];  // empty unless the tuple is live
                    }
                    if constexpr (EB == 4) {
                        // the first two passes run without the warp vote: of 128
                        // tuples some are nearly always left after them (2^27 x
                        // 2^27 int32 join 1.030 -> 1.023 ms; the same for 8-byte
                        // entries measured 1.97 -> 2.14 ms and is not used there)
#pragma unroll
                        for (int pass = 0; pass < 2; ++pass)
#pragma unroll
                            for (int u = 0; u < U; ++u) walk_exact4(at[u], end[u], fqs[u], lim);
                        for (;;) {
                            bool more = false;
#pragma unroll
                            for (int u = 0; u < U; ++u) more = more || at[u] < end[u];
                            if (!__any_sync(0xffffffffu, more)) break;
#pragma unroll
                            for (int u = 0; u < U; ++u) walk_exact4(at[u], end[u], fqs[u], lim);
                        }
                    } else {
                        for (;;) {
                            bool more = false;
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                walk_exact8(at[u], end[u], fqs[u], lim, ExactEntry<K>::key_lo(k[u]));
                                more = more || at[u] < end[u];
                            }
                            if (!__any_sync(0xffffffffu, more)) break;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        emit[u] = at[u] > end[u];  // a match stopped the cursor past its end
                        brow[u] = walk_row(at[u], end[u]) & x_rmask;
                    }
                    append_direct(emit, brow, r);
                } else if constexpr (UNIQUE && TABLE == TABLE_BUCKET) {
                    // every tuple matches at most once: the predicated walk of
                    // the EXACT case over {key, row} entries
                    if constexpr (Entry<K>::BYTES == 8) {
                        const uint32_t tb = static_cast<uint32_t>(__cvta_generic_to_shared(table));
                        bool emit[U];
                        uint32_t brow[U], at[U], end[U];
                        const uint16_t* e16 = reinterpret_cast<const uint16_t*>(ends);
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const bool ok = r[u] >= 0 && in_piece(h[u]);
                            const uint32_t b = bucket_of(h[u]);
                            const uint32_t e_lo = e16[b], e_hi = e16[b + 1];
                            at[u] = tb + e_lo * 8u;
                            end[u] = ok ? tb + e_hi * 8u : at[u];
                        }
                        for (;;) {
                            bool more = false;
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                walk_bucket8(at[u], end[u], static_cast<uint32_t>(k[u]));
                                more = more || at[u] < end[u];
                            }
                            if (!__any_sync(0xffffffffu, more)) break;
                        }
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            emit[u] = at[u] > end[u];
                            brow[u] = walk_row(at[u], end[u]);
                        }
                        append_direct(emit, brow, r);
                    } else {  // 12-byte entries {key, row} of 8-byte keys
                        bool emit[U];
                        uint32_t brow[U];
                        int at[U], end[U];
                        const uint16_t* e16 = reinterpret_cast<const uint16_t*>(ends);
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            emit[u] = false;
                            brow[u] = 0;
                            const bool ok = r[u] >= 0 && in_piece(h[u]);
                            const uint32_t b = bucket_of(h[u]);
                            const int e_lo = e16[b], e_hi = e16[b + 1];
                            at[u] = ok ? e_lo : 0;
                            end[u] = ok ? e_hi : 0;
                        }
                        for (;;) {
                            bool more = false;
#pragma unroll
                            for (int u = 0; u < U; ++u) {
                                const bool act = at[u] < end[u];
                                Cmp ek;
                                uint32_t er;
                                E::get(table, act ? at[u] : 0, ek, er);
                                const bool hit = act && ek == k[u];
                                brow[u] = hit ? er : brow[u];
                                emit[u] = emit[u] || hit;
                                at[u] = hit ? end[u] : at[u] + (act ? 1 : 0);
                                more = more || at[u] < end[u];
                            }
                            if (!__any_sync(0xffffffffu, more)) break;
                        }
                        append_direct(emit, brow, r);
                    }
                } else if constexpr (UNIQUE) {
                    // every tuple matches at most once: one lookup, one append per warp step
                    bool emit[U];
                    uint32_t brow[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        emit[u] = false;
                        brow[u] = 0;
                        if (r[u] >= 0 && in_piece(h[u])) {
                            int at_u = 0, end_u = 0, steps_u = 0;
                            uint32_t sl_u = 0;
                            bool live_u = true;
                            start(u, at_u, end_u, sl_u);
                            emit[u] = lookup(u, at_u, end_u, sl_u, steps_u, live_u, brow[u]);
                        }
                    }
                    append_direct(emit, brow, r);
                } else {
                    // repeated build keys: every tuple walks on, one match per lane per append
                    bool live[U], emit[U];
                    uint32_t brow[U], sl[U];
                    int at[U], end[U], steps[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        live[u] = r[u] >= 0 && in_piece(h[u]);
                        at[u] = end[u] = steps[u] = 0;
                        sl[u] = 0;
                        brow[u] = 0;
                        if (live[u]) start(u, at[u], end[u], sl[u]);
                    }
                    for (;;) {
                        bool any_live = false;
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            emit[u] = live[u] && lookup(u, at[u], end[u], sl[u], steps[u], live[u], brow[u]);
                            any_live |= live[u];
                        }
                        append_direct(emit, brow, r);
                        if (!__any_sync(0xffffffffu, any_live)) break;
                    }
                }
                s0 = s_after;
            }
        }
    }
    // ---- record this CTA's entries and last chunk for the fix-up ----
    __syncthreads();
    if (!BATCH && threadIdx.x == 0) {
        const uint32_t q = s_q;
        a.cta_q[blockIdx.x] = q;
        a.cta_last[blockIdx.x] =
            (q > 0 && write_out) ? static_cast<int64_t>(s_cslot[((q - 1) / OUT_CHUNK) % OUT_SLOTS] & ((1ull << 40) - 1))
                                 : -1;
    }
}

// ---------------------------------------------------------------------------
// Fix-up of the output.  The CTAs' reservations cover [0, reserved); CTA c
// used the first cta_q[c] % OUT_CHUNK entries of its last chunk, so the
// rest of that chunk is a gap.  total = sum cta_q.  Every gap position below
// total is filled with a valid entry from at or above total (those lie in
// [total, reserved) outside the gaps), in order: no two moves touch the
// same position and sources never overlap destinations.
// Plan (one CTA): sorted gaps -> hole segments (< total) and mover
// segments (>= total), their prefix sums; *count = total.
// seg layout: [0] = n_holes, [1] = n_movers, [2] = moves; then
// hole (start, prefix) pairs, then mover (start, prefix) pairs.
constexpr int MAX_FIXUP_CTAS = 1024;  // join CTAs one fix-up plan covers: one thread (and gap) each

// Exclusive prefix over the block of one value per thread; the block's
// total goes to *total (every thread).  Contains two barriers.
__device__ __forceinline__ long long block_excl_scan(long long v, long long* s_w, long long* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    long long incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    long long before = 0, all = 0;
    for (int w = 0; w < nw; ++w) {
        before += w < warp ? s_w[w] : 0;
        all += s_w[w];
    }
    *total = all;
    __syncthreads();  // s_w is free again
    return before + incl - v;
}

// One block of at least n_cta threads (a multiple of 32).  Thread c takes
// CTA c's gap (the unused tail of its last chunk); the gaps are ranked by
// start, and thread g then works out the hole below the true total that
// gap g leaves and the stretch of entries at or above the total that ends
// at it; block scans number both lists.  The stretch after the last gap is
// thread 0's.
__global__ void __launch_bounds__(MAX_FIXUP_CTAS) join_fixup_plan_kernel(const int64_t* __restrict__ cta_q,
                                                               const int64_t* __restrict__ cta_last, int32_t n_cta,
                                                               unsigned long long* count,
                                                               const unsigned long long* __restrict__ base_count,
                                                               int64_t capacity,
                                                               int32_t write_out, int64_t* __restrict__ seg,
                                                               uint32_t* __restrict__ status)
{
    __shared__ long long g_at[MAX_FIXUP_CTAS];                        // gap start by CTA (-1: none)
    __shared__ long long g_start[MAX_FIXUP_CTAS], g_end[MAX_FIXUP_CTAS];  // gaps by rank
    __shared__ long long s_w[32];
    const int t = threadIdx.x;
    if (n_cta > static_cast<int>(blockDim.x)) {  // gaps of CTAs past the block would stay unfilled
        if (t == 0) raise_status(status, ST_INTERNAL);
        return;
    }
    long long q = 0, gs = -1, ge = -1;
    if (t < n_cta) {
        q = cta_q[t];
        const long long rem = q % OUT_CHUNK;
        if (write_out && q > 0 && rem != 0 && cta_last[t] >= 0) {
            gs = cta_last[t] + rem;
            ge = cta_last[t] + OUT_CHUNK;
        }
    }
    g_at[t] = gs;
    long long sum, ng;
    block_excl_scan(q, s_w, &sum);  // its barriers also publish g_at
    const long long total = sum + (base_count ? static_cast<long long>(*base_count) : 0);
    const long long reserved = static_cast<long long>(*count);
    // rank by start: starts are distinct positions of distinct chunks
    if (gs >= 0) {
        int rank = 0;
        for (int c = 0; c < n_cta; ++c) rank += (g_at[c] >= 0 && g_at[c] < gs) ? 1 : 0;
        g_start[rank] = gs;
        g_end[rank] = ge;
    }
    block_excl_scan(gs >= 0 ? 1 : 0, s_w, &ng);  // and publish the ranked gaps
    const bool lists = write_out && total <= capacity;
    long long h_len = 0, m_lo = 0, m_len = 0, h_at = 0;
    if (lists && t < ng) {
        h_at = g_start[t];
        const long long h_end = g_end[t];
        if (h_at < total) h_len = (h_end < total ? h_end : total) - h_at;
        // entries from the previous gap's end (or 0) up to this gap, at or above the total
        const long long prev = t > 0 ? g_end[t - 1] : 0;
        m_lo = prev > total ? prev : total;
        const long long hi = h_at < reserved ? h_at : reserved;
        m_len = hi > m_lo ? hi - m_lo : 0;
    }
    long long nh, hp, nm, mp;
    const long long h_idx = block_excl_scan(h_len > 0 ? 1 : 0, s_w, &nh);
    const long long h_pre = block_excl_scan(h_len, s_w, &hp);
    const long long m_idx = block_excl_scan(m_len > 0 ? 1 : 0, s_w, &nm);
    const long long m_pre = block_excl_scan(m_len, s_w, &mp);
    int64_t* hole = seg + 4;
    int64_t* mover = seg + 4 + 2 * (n_cta + 2);
    if (h_len > 0) {
        hole[2 * h_idx] = h_at;
        hole[2 * h_idx + 1] = h_pre;
    }
    if (m_len > 0) {
        mover[2 * m_idx] = m_lo;
        mover[2 * m_idx + 1] = m_pre;
    }
    if (t == 0) {
        *count = static_cast<unsigned long long>(total);
        long long moves = 0;
        if (lists) {
            // the entries after the last gap
            const long long last = ng > 0 ? g_end[ng - 1] : 0;
            const long long lo = last > total ? last : total;
            if (reserved > lo) {
                mover[2 * nm] = lo;
                mover[2 * nm + 1] = mp;
                mp += reserved - lo;
                ++nm;
            }
            if (hp != mp) raise_status(status, ST_INTERNAL);
            moves = hp < mp ? hp : mp;
        } else if (write_out) {
            raise_status(status, ST_CAPACITY);
            nh = nm = 0;
        } else {
            nh = nm = 0;
        }
        seg[0] = nh;
        seg[1] = nm;
        seg[2] = moves;
    }
}

__device__ __forceinline__ int seg_find(const int64_t* s, int n, long long i)
{
    int lo = 0, hi = n;  // last segment with prefix <= i
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s[2 * mid + 1] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void join_fixup_move_kernel(const int64_t* __restrict__ seg, int32_t n_cta, int32_t* out_build,
                                       int32_t* out_probe, int64_t capacity, const int32_t* __restrict__ over_build,
                                       const int32_t* __restrict__ over_probe)
{
    const int nh = static_cast<int>(seg[0]), nm = static_cast<int>(seg[1]);
    const long long moves = seg[2];
    const int64_t* hole = seg + 4;
    const int64_t* mover = seg + 4 + 2 * (n_cta + 2);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < moves;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int h = seg_find(hole, nh, i), m = seg_find(mover, nm, i);
        const long long dst = hole[2 * h] + (i - hole[2 * h + 1]);
        const long long src = mover[2 * m] + (i - mover[2 * m + 1]);
        int32_t b, q;
        if (src < capacity) {
            b = out_build[src];
            q = out_probe[src];
        } else {
            b = over_build[src - capacity];
            q = over_probe[src - capacity];
        }
        out_build[dst] = b;
        out_probe[dst] = q;
    }
}

}  // namespace pj
