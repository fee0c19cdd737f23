// pj_join.cuh -- per-partition shared-memory hash build and probe.
//
// Reference counterparts: hash_join (hash_join_kernels.cuh:24-200), the
// work split of handle_skewed_data (skewed_data_handler.cuh:21-91) and the
// launch of shared_memory_hash_join (partitioned_join.cuh:178-251).
//
// Work items.  Partition p with b build and q probe tuples (padded ranges
// from the scatter) becomes S_p x K_p items: S_p splits the build side so
// that each piece fits one table (by hash bits, or by position as the
// reference does), K_p = ceil(q / probe_chunk) splits the probe side (the
// reference has no probe split, so one CTA walks a hot partition's whole
// probe run).  Items are numbered partition-major, then probe chunk, then
// build split, so the CTAs that share a probe chunk run side by side and
// read it from L2.  A persistent grid claims items through an atomic
// counter.
//
// Table.  Open addressing with linear probing, table_slots slots of
// {key, row}; row == -1 marks an empty slot, so every key value (the
// reference's -1 sentinel included) joins.  Inserts claim a slot with a CAS
// on the row word.  The slot of a key is PJ_SLOT_FAST (multiply-high of the
// hash bits that digits and splits did not consume) or PJ_SLOT_REF
// (abs((int)h % T), hash_join_kernels.cuh:100-101).
//
// Output.  Matches are appended to a shared-memory buffer with one shared
// atomic per warp (ballot + popc); when the buffer passes its high-water
// mark the CTA reserves room in the output with ONE global atomicAdd and
// copies the buffer out coalesced (the reference's write_back_buffer,
// hash_join_kernels.cuh:150-199, does a global atomic per overflowing match).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_bulk.cuh"
#include "pj_device.cuh"

namespace pj {

constexpr uint32_t EMPTY_ROW = 0xffffffffu;

struct JoinArgs {
    const uint32_t* build_tuples;
    const uint32_t* probe_tuples;
    const int64_t* build_off;   // partition p = [build_off[p*b_items], build_off[(p+1)*b_items])
    const int64_t* probe_off;
    int32_t b_items;
    int32_t p_items;
    int32_t P;
    int32_t digit_bits;         // top hash bits consumed by partition digits (HASH digits), else 0
    const int32_t* split_log2;  // per partition: log2 S_p (hash split) or S_p (position split)
    const int64_t* item_off;    // exclusive scan of items per partition, P+1 entries
    uint32_t* queue;            // item counter (zeroed)
    int32_t table_slots;
    int32_t probe_chunk;        // tuples
    int32_t position_chunk;     // build tuples per position split piece
    int32_t* out_build;
    int32_t* out_probe;
    int64_t capacity;
    unsigned long long* count;  // device int64 match counter
    uint32_t* status;
};

// Items per partition (S_p x K_p) and the split of partition p.
__global__ void join_items_kernel(const int64_t* __restrict__ build_off, const int64_t* __restrict__ probe_off,
                                  int32_t b_items, int32_t p_items, int32_t P,
                                  const int32_t* __restrict__ build_tot, const int32_t* __restrict__ probe_tot,
                                  int32_t cap_per_table, int32_t probe_chunk, int32_t hash_split,
                                  int32_t max_split_log2, int32_t* __restrict__ split_out,
                                  int64_t* __restrict__ items_out, uint32_t* __restrict__ status)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int64_t bc = build_tot[p], pc = probe_tot[p];
    const int64_t prange = probe_off[static_cast<int64_t>(p + 1) * p_items] - probe_off[static_cast<int64_t>(p) * p_items];
    int64_t items = 0;
    int32_t split = 0;
    if (bc > 0 && pc > 0) {
        int64_t S;
        if (hash_split) {
            int lg = 0;
            while (lg < max_split_log2 && (bc + (1ll << lg) - 1) / (1ll << lg) > cap_per_table) ++lg;
            split = lg;
            S = 1ll << lg;
        } else {
            S = (bc + cap_per_table - 1) / cap_per_table;
            if (S < 1) S = 1;
            split = static_cast<int32_t>(S);
        }
        const int64_t K = (prange + probe_chunk - 1) / probe_chunk;
        items = S * K;
    }
    split_out[p] = split;
    items_out[p] = items;
}

template <typename K> struct TableSlot;

// 4-byte keys: one 8-byte slot {key, row} -> one shared load per step.
template <> struct TableSlot<int32_t> {
    static constexpr int BYTES = 8;
    uint2* s;
    __device__ __forceinline__ void bind(uint8_t* base, int T) { (void)T; s = reinterpret_cast<uint2*>(base); }
    __device__ __forceinline__ void clear(int i) { s[i] = make_uint2(0u, EMPTY_ROW); }
    __device__ __forceinline__ bool try_claim(int i, int32_t key, int32_t row)
    {
        if (atomicCAS(&s[i].y, EMPTY_ROW, static_cast<uint32_t>(row)) == EMPTY_ROW) {
            s[i].x = static_cast<uint32_t>(key);
            return true;
        }
        return false;
    }
    // returns row, or EMPTY_ROW; sets hit if the key matches
    __device__ __forceinline__ uint32_t look(int i, int32_t key, bool& hit) const
    {
        const uint2 v = s[i];
        hit = v.y != EMPTY_ROW && static_cast<int32_t>(v.x) == key;
        return v.y;
    }
};

// 8-byte keys: keys[T] then rows[T] (12 bytes a slot).
template <> struct TableSlot<int64_t> {
    static constexpr int BYTES = 12;
    unsigned long long* k;
    uint32_t* r;
    __device__ __forceinline__ void bind(uint8_t* base, int T)
    {
        k = reinterpret_cast<unsigned long long*>(base);
        r = reinterpret_cast<uint32_t*>(base + static_cast<size_t>(T) * 8);
    }
    __device__ __forceinline__ void clear(int i) { r[i] = EMPTY_ROW; }
    __device__ __forceinline__ bool try_claim(int i, int64_t key, int32_t row)
    {
        if (atomicCAS(&r[i], EMPTY_ROW, static_cast<uint32_t>(row)) == EMPTY_ROW) {
            k[i] = static_cast<unsigned long long>(key);
            return true;
        }
        return false;
    }
    __device__ __forceinline__ uint32_t look(int i, int64_t key, bool& hit) const
    {
        const uint32_t row = r[i];
        hit = row != EMPTY_ROW && static_cast<int64_t>(k[i]) == key;
        return row;
    }
};

template <typename K>
__device__ __forceinline__ void smem_tuple(const uint8_t* stage, int j, K& key, int32_t& row);

template <>
__device__ __forceinline__ void smem_tuple<int32_t>(const uint8_t* stage, int j, int32_t& key, int32_t& row)
{
    const uint2 v = reinterpret_cast<const uint2*>(stage)[j];
    key = static_cast<int32_t>(v.x);
    row = static_cast<int32_t>(v.y);
}

template <>
__device__ __forceinline__ void smem_tuple<int64_t>(const uint8_t* stage, int j, int64_t& key, int32_t& row)
{
    const uint32_t* w = reinterpret_cast<const uint32_t*>(stage) + 3 * j;
    key = static_cast<int64_t>((static_cast<uint64_t>(w[1]) << 32) | w[0]);
    row = static_cast<int32_t>(w[2]);
}

template <typename K, int THREADS, int OB, int NSTAGE, int STAGE_TUPLES>
struct JoinSmem {
    static constexpr int TB = TupleTraits<K>::WORDS * 4;
    static constexpr int STAGE_BYTES = STAGE_TUPLES * TB;
    static size_t bytes(int T)
    {
        const size_t table = (static_cast<size_t>(T) * TableSlot<K>::BYTES + 127) & ~size_t(127);
        return static_cast<size_t>(NSTAGE) * STAGE_BYTES + static_cast<size_t>(OB) * 8 + table;
    }
};

__device__ __forceinline__ int upper_bound_i64(const int64_t* a, int n, int64_t x)
{
    int lo = 0, hi = n;  // first index with a[i] > x
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <typename K, bool UNIQUE, bool HASH_SPLIT, bool SLOT_REF, int THREADS, int OB, int NSTAGE,
          int STAGE_TUPLES>
__global__ void __launch_bounds__(THREADS, 1) join_kernel(JoinArgs a)
{
    using SM = JoinSmem<K, THREADS, OB, NSTAGE, STAGE_TUPLES>;
    static_assert(STAGE_TUPLES % THREADS == 0, "a stage holds whole rounds");
    static_assert(OB >= 2 * THREADS, "output buffer needs a round of headroom");
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* stages = smem;
    int32_t* ob_b = reinterpret_cast<int32_t*>(smem + NSTAGE * SM::STAGE_BYTES);
    int32_t* ob_p = ob_b + OB;
    TableSlot<K> table;
    table.bind(reinterpret_cast<uint8_t*>(ob_p + OB), a.table_slots);
    __shared__ uint64_t bars[NSTAGE];
    __shared__ int64_t s_item;
    __shared__ int s_obn;
    __shared__ unsigned long long s_gpos;

    const int T = a.table_slots;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    BulkRing<NSTAGE, SM::STAGE_BYTES> ring;
    ring.stages = stages;
    ring.bars = bars;
    ring.phase_bits = 0;
    ring.init_barriers();
    if (threadIdx.x == 0) s_obn = 0;
    const int64_t total_items = a.item_off[a.P];

    auto flush = [&]() {
        if (threadIdx.x == 0) s_gpos = atomicAdd(a.count, static_cast<unsigned long long>(s_obn));
        __syncthreads();
        const int n = s_obn;
        const int64_t g = static_cast<int64_t>(s_gpos);
        if (g + n > a.capacity && threadIdx.x == 0) raise_status(a.status, ST_CAPACITY);
        for (int i = threadIdx.x; i < n; i += THREADS) {
            if (g + i < a.capacity) {
                a.out_build[g + i] = ob_b[i];
                a.out_probe[g + i] = ob_p[i];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_obn = 0;
        __syncthreads();
    };

    for (;;) {
        if (threadIdx.x == 0) s_item = static_cast<int64_t>(atomicAdd(a.queue, 1u));
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total_items) break;
        const int p = upper_bound_i64(a.item_off, a.P + 1, item) - 1;
        const int64_t local = item - a.item_off[p];
        const int32_t split = a.split_log2[p];
        const int64_t S = HASH_SPLIT ? (1ll << split) : split;
        const int64_t piece = local % S;
        const int64_t pchunk = local / S;
        const int sbits = HASH_SPLIT ? split : 0;
        const int skip = a.digit_bits + sbits;

        const int64_t b_lo0 = a.build_off[static_cast<int64_t>(p) * a.b_items];
        const int64_t b_hi0 = a.build_off[static_cast<int64_t>(p + 1) * a.b_items];
        int64_t b_lo = b_lo0, b_hi = b_hi0;
        if (!HASH_SPLIT) {
            // position pieces of position_chunk tuples, rounded to 16-byte multiples
            b_lo = b_lo0 + piece * a.position_chunk;
            b_hi = b_lo + a.position_chunk < b_hi0 ? b_lo + a.position_chunk : b_hi0;
            if (b_lo > b_hi) b_lo = b_hi;
        }
        const int64_t q_lo0 = a.probe_off[static_cast<int64_t>(p) * a.p_items];
        const int64_t q_hi0 = a.probe_off[static_cast<int64_t>(p + 1) * a.p_items];
        const int64_t q_lo = q_lo0 + pchunk * a.probe_chunk;
        const int64_t q_hi = q_lo + a.probe_chunk < q_hi0 ? q_lo + a.probe_chunk : q_hi0;

        // the sbits hash bits just below the digit bits select the piece
        const int piece_shift = 32 - (sbits > 0 ? sbits : 1);
        auto in_piece = [&](uint32_t h) -> bool {
            if (!HASH_SPLIT || sbits == 0) return true;
            return static_cast<int64_t>((h << a.digit_bits) >> piece_shift) == piece;
        };
        auto slot_of = [&](uint32_t h) -> int {
            return SLOT_REF ? static_cast<int>(slot_ref(h, T)) : static_cast<int>(slot_fast(h, skip, T));
        };

        for (int i = threadIdx.x; i < T; i += THREADS) table.clear(i);
        __syncthreads();

        // ---- build ----
        ring.start(a.build_tuples + (b_lo * SM::TB) / 4, (b_hi - b_lo) * SM::TB, a.status);
        {
            const int64_t nch = ring.num_chunks();
            for (int64_t c = 0; c < nch; ++c) {
                const uint8_t* st = ring.wait(c);
                const int64_t left = (b_hi - b_lo) - c * STAGE_TUPLES;
                const int cnt = left < STAGE_TUPLES ? static_cast<int>(left) : STAGE_TUPLES;
                for (int j = threadIdx.x; j < cnt; j += THREADS) {
                    K key;
                    int32_t row;
                    smem_tuple<K>(st, j, key, row);
                    if (row < 0) continue;
                    const uint32_t h = hash_key(key);
                    if (!in_piece(h)) continue;
                    int sl = slot_of(h);
                    int tries = 0;
                    while (!table.try_claim(sl, key, row)) {
                        if (++sl == T) sl = 0;
                        if (++tries >= T) {
                            raise_status(a.status, ST_OVERFLOW);
                            break;
                        }
                    }
                }
                __syncthreads();
                ring.release(c);
            }
        }
        __syncthreads();

        // ---- probe ----
        ring.start(a.probe_tuples + (q_lo * SM::TB) / 4, (q_hi - q_lo) * SM::TB, a.status);
        {
            const int64_t nch = ring.num_chunks();
            for (int64_t c = 0; c < nch; ++c) {
                const uint8_t* st = ring.wait(c);
                const int64_t left = (q_hi - q_lo) - c * STAGE_TUPLES;
                const int cnt = left < STAGE_TUPLES ? static_cast<int>(left) : STAGE_TUPLES;
                const int64_t row_base = 0;
                (void)row_base;
                for (int r0 = 0; r0 < cnt; r0 += THREADS) {
                    const int j = r0 + threadIdx.x;
                    K key = K(0);
                    int32_t prow = -1;
                    bool pending = false;
                    int sl = 0, steps = 0;
                    if (j < cnt) {
                        smem_tuple<K>(st, j, key, prow);
                        if (prow >= 0) {
                            const uint32_t h = hash_key(key);
                            if (in_piece(h)) {
                                pending = true;
                                sl = slot_of(h);
                            }
                        }
                    }
                    bool more;
                    do {
                        // walk to the next match (or an empty slot)
                        bool emit = false;
                        uint32_t brow = 0;
                        while (pending) {
                            bool hit;
                            const uint32_t rw = table.look(sl, key, hit);
                            if (rw == EMPTY_ROW) { pending = false; break; }
                            if (++sl == T) sl = 0;
                            if (++steps > T) { pending = false; break; }
                            if (hit) {
                                emit = true;
                                brow = rw;
                                if (UNIQUE) pending = false;
                                break;
                            }
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, emit);
                        if (m) {
                            const int leader = __ffs(m) - 1;
                            int base = 0;
                            if (lane == leader) base = atomicAdd(&s_obn, __popc(m));
                            base = __shfl_sync(0xffffffffu, base, leader);
                            if (emit) {
                                const int at = base + __popc(m & lt_mask);
                                ob_b[at] = static_cast<int32_t>(brow);
                                ob_p[at] = prow;
                            }
                        }
                        more = __syncthreads_or(pending) != 0;
                        if (s_obn > OB - THREADS) flush();
                    } while (more);
                }
                __syncthreads();
                ring.release(c);
            }
        }
        __syncthreads();
    }
    if (s_obn > 0) flush();
}

}  // namespace pj
