// pj_partition.cuh -- radix histogram, decoupled look-back scan and
// write-combining scatter.
//
// Layout of one partitioned column.  The input is cut into n_items equal
// chunks ("items", one per resident scatter CTA).  Item i's tuples of
// partition p form the segment [off[p*n_items + i], off[p*n_items + i + 1])
// of the output, where off is the exclusive scan of the per-(p, i) counts,
// each rounded up to W tuples.  So partitions are contiguous
// (partition p = [off[p*n_items], off[(p+1)*n_items]) ), every segment starts
// on a W-tuple boundary, and the padding tuples that fill a segment's last
// W-group carry row = -1.
//
// Tuples.  4-byte keys are stored as {murmur(key), row}: MurmurHash3_x86_32
// of a 4-byte key is a bijection of 32-bit values (every step -- odd
// multiplies, rotations, xor/add of constants, the fmix32 xor-shifts -- is
// invertible), so equal hashes mean equal keys and the join never hashes
// again.  8-byte keys are stored as {key_lo, key_hi, murmur(key), row}.
//
// Reference counterparts: histogram_pass_one (partition_kernels.cuh:141-194),
// the ExclusiveSum + copy of partitioned_join.cuh:86-88, partition_pass_one
// (partition_kernels.cuh:197-326).  The reference stages an 8 192-key tile in
// shared memory and flushes each partition's run with 32 threads; here each
// CTA keeps a W-tuple write-combining buffer per partition and writes only
// whole, aligned W-tuple groups (32-byte sectors), so the fan-out of one pass
// reaches 4 096.
//
// With the heavy-key path (pj_heavy.cuh) the probe side's histogram skips
// heavy keys and its scatter writes their output pairs directly.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_device.cuh"
#include "pj_heavy.cuh"
#include "pj_types.cuh"

namespace pj {

template <typename K>
__device__ __forceinline__ uint32_t key_digit(const DigitFn& f, K key)
{
    return digit_of(f, key, f.mode == 1 ? hash_key(key) : 0u);
}

// Elements of a 16-byte vector.
template <typename K> struct Vec16 { static constexpr int N = 16 / sizeof(K); };

template <typename K>
__device__ __forceinline__ void load_vec16(const K* p, K (&out)[Vec16<K>::N])
{
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    if constexpr (sizeof(K) == 4) {
        out[0] = static_cast<K>(v.x); out[1] = static_cast<K>(v.y);
        out[2] = static_cast<K>(v.z); out[3] = static_cast<K>(v.w);
    } else {
        out[0] = static_cast<K>((static_cast<uint64_t>(v.y) << 32) | v.x);
        out[1] = static_cast<K>((static_cast<uint64_t>(v.w) << 32) | v.z);
    }
}

// Byte offset of the heavy table in the scatter's shared memory: after P
// buffers of capw words, P fill counts and P cursors, rounded up to 16 bytes.
__host__ __device__ constexpr size_t heavy_table_offset(int P, int capw)
{
    return (static_cast<size_t>(P) * capw * 4 + static_cast<size_t>(P) * 8 + 15) & ~static_cast<size_t>(15);
}

// Output of heavy probe keys (heavy-key path).  The probe histogram counts,
// per item, the heavy probe rows that have a build row; item i's pairs then
// go to [sum of the counts of items < i, ...) -- exact positions, no global
// atomics -- and the join's output starts after all of them.
struct HeavyOut {
    const int32_t* heavy_row;          // build row of each heavy key (-1: none)
    unsigned long long* item_count;    // per scatter item: heavy pairs (zeroed by the caller)
    int32_t* out_build;                // nullptr: count only
    int32_t* out_probe;
    int64_t capacity;
};

// ---------------------------------------------------------------------------
// Histogram.  Grid = n_items * hsplit CTAs; CTA c counts the keys of the
// (c % hsplit)-th slice of item c / hsplit's chunk in shared memory and adds
// them into counts_T[p*n_items + item] (zeroed by the caller) and totals[p].
constexpr int HIST_THREADS = 512;
constexpr int HIST_UNROLL = 4;  // 16-byte vectors in flight per thread

template <typename K, bool HASHD, bool HEAVY>
__global__ void __launch_bounds__(HIST_THREADS) hist_keys_kernel(const K* __restrict__ keys, int64_t n,
                                                                 int64_t chunk, int32_t n_items, int32_t hsplit,
                                                                 DigitFn f, int32_t P,
                                                                 uint32_t* __restrict__ counts_T,
                                                                 int32_t* __restrict__ totals,
                                                                 typename HeavyArg<HEAVY>::type hs, HeavyOut ho)
{
    constexpr int VN = Vec16<K>::N;
    extern __shared__ __align__(16) uint32_t cnt[];
    const int item = blockIdx.x / hsplit, part = blockIdx.x % hsplit;
    for (int p = threadIdx.x; p < P; p += HIST_THREADS) cnt[p] = 0;
    HeavyTable heavy;
    uint32_t heavy_hits = 0;
    if constexpr (HEAVY) {
        heavy.bind(reinterpret_cast<uint8_t*>(cnt + ((P + 3) & ~3)));
        heavy.build<K>(hs, ho.heavy_row);  // ends with a barrier
    }
    __syncthreads();
    int64_t lo = static_cast<int64_t>(item) * chunk;
    int64_t hi = lo + chunk < n ? lo + chunk : n;
    if (lo > hi) lo = hi;
    // this CTA's slice of the item, 16-element aligned
    const int64_t per = (((hi - lo) + hsplit - 1) / hsplit + 15) & ~int64_t(15);
    int64_t s_lo = lo + part * per;
    int64_t s_hi = s_lo + per < hi ? s_lo + per : hi;
    if (s_lo > s_hi) s_lo = s_hi;
    // digit of key k, or -1 for a heavy probe key (not partitioned)
    auto digit = [&](K k) -> int {
        if constexpr (HEAVY) {
            const HeavyHit e = heavy.find(k);
            if (e.idx >= 0) {
                heavy_hits += e.row >= 0 ? 1u : 0u;
                return -1;
            }
        }
        uint32_t h = 0;
        if constexpr (HASHD) h = hash_key(k);
        return static_cast<int>(HASHD ? ((h >> f.shift) & f.mask)
                                      : (static_cast<uint32_t>(static_cast<uint64_t>(k) >> f.shift) & f.mask));
    };
    auto count = [&](K k) {
        const int d = digit(k);
        if (d >= 0) atomicAdd(&cnt[d], 1u);
    };
    constexpr int STEP = HIST_THREADS * VN * HIST_UNROLL;
    int64_t base = s_lo;
    // the next step's vectors load while this step's keys are counted
    K v[HIST_UNROLL][VN];
    auto load_step = [&](int64_t at) {
#pragma unroll
        for (int u = 0; u < HIST_UNROLL; ++u)
            load_vec16<K>(keys + at + (static_cast<int64_t>(u) * HIST_THREADS + threadIdx.x) * VN, v[u]);
    };
    if (base + STEP <= s_hi) load_step(base);
    for (; base + STEP <= s_hi; base += STEP) {
        K c[HIST_UNROLL][VN];
#pragma unroll
        for (int u = 0; u < HIST_UNROLL; ++u)
#pragma unroll
            for (int e = 0; e < VN; ++e) c[u][e] = v[u][e];
        if (base + 2 * STEP <= s_hi) load_step(base + STEP);
#pragma unroll
        for (int u = 0; u < HIST_UNROLL; ++u)
#pragma unroll
            for (int e = 0; e < VN; ++e) count(c[u][e]);
    }
    for (int64_t i = base + threadIdx.x; i < s_hi; i += HIST_THREADS) count(keys[i]);
    if constexpr (HEAVY) {
        heavy_hits = __reduce_add_sync(0xffffffffu, heavy_hits);
        if ((threadIdx.x & 31) == 0 && heavy_hits) atomicAdd(&ho.item_count[item], static_cast<unsigned long long>(heavy_hits));
    }
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += HIST_THREADS) {
        const uint32_t c = cnt[p];
        if (c) {
            atomicAdd(&counts_T[static_cast<int64_t>(p) * n_items + item], c);
            if (totals != nullptr) atomicAdd(&totals[p], static_cast<int32_t>(c));
        }
    }
}

// Global digit histogram (no per-item split): the stage entry point
// pj_radix_histogram and the exact planner.
template <typename K>
__global__ void __launch_bounds__(512) global_hist_kernel(const K* __restrict__ keys, int64_t n, DigitFn f,
                                                          int32_t P, int32_t* __restrict__ hist)
{
    extern __shared__ __align__(16) uint32_t sh_hist[];
    for (int p = threadIdx.x; p < P; p += blockDim.x) sh_hist[p] = 0;
    __syncthreads();
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        atomicAdd(&sh_hist[key_digit(f, keys[i])], 1u);
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x)
        if (sh_hist[p]) atomicAdd(&hist[p], static_cast<int32_t>(sh_hist[p]));
}

// ---------------------------------------------------------------------------
// Single-pass exclusive scan with decoupled look-back (Merrill & Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016).
// out[i] = sum_{j<i} r(in[j]), out[m] = total, with r(x) = x rounded up to a
// multiple of round_to.  Tiles are claimed through an atomic counter, so a
// tile's predecessors are always already running; the look-back spin is
// bounded all the same.  tile_state and tile_counter must be zero.
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr uint64_t TS_AGG = 1ull << 62;
constexpr uint64_t TS_PREFIX = 2ull << 62;
constexpr uint64_t TS_VALUE = (1ull << 62) - 1;

__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// The look-back wait of a scan: how many polls a tile makes before it gives
// up (ST_TIMEOUT), and a tile that never publishes (-1: none).  Joins use
// {-1, SPIN_LIMIT}; pj_diag_scan_timeout withholds a tile to show that a
// wait which never ends returns an error instead of hanging.
struct ScanWait {
    int64_t withhold_tile;
    uint32_t spin_limit;
};

template <typename TIn>
__global__ void __launch_bounds__(SCAN_THREADS) lookback_scan_kernel(const TIn* __restrict__ in, int64_t m,
                                                                     uint32_t round_to, int64_t* __restrict__ out,
                                                                     uint64_t* __restrict__ tile_state,
                                                                     uint32_t* __restrict__ tile_counter,
                                                                     uint32_t* __restrict__ status, ScanWait wait)
{
    __shared__ uint32_t s_tile;
    __shared__ int64_t s_warp[SCAN_THREADS / 32];
    __shared__ int64_t s_excl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const int64_t tile = s_tile;
    const int64_t ntiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    const int64_t base = tile * SCAN_TILE + static_cast<int64_t>(threadIdx.x) * SCAN_ITEMS;

    int64_t v[SCAN_ITEMS];
    int64_t sum = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        const int64_t idx = base + j;
        int64_t x = idx < m ? static_cast<int64_t>(in[idx]) : 0;
        if (round_to > 1) x = (x + round_to - 1) / round_to * round_to;
        v[j] = x;
        sum += x;
    }
    int64_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) s_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const int64_t block_total = s_warp[SCAN_THREADS / 32 - 1];
    const int64_t thread_excl = incl - sum + (warp > 0 ? s_warp[warp - 1] : 0);

    if (threadIdx.x == 0) {
        int64_t excl = 0;
        if (tile == wait.withhold_tile) {
            // publishes nothing: its successors' waits run out
        } else if (tile == 0) {
            st_release_u64(&tile_state[0], TS_PREFIX | static_cast<uint64_t>(block_total));
        } else {
            st_release_u64(&tile_state[tile], TS_AGG | static_cast<uint64_t>(block_total));
            int64_t i = tile - 1;
            uint32_t spins = 0;
            while (i >= 0) {
                const uint64_t s = ld_acquire_u64(&tile_state[i]);
                const uint64_t flag = s & ~TS_VALUE;
                if (flag == 0) {
                    if (++spins > wait.spin_limit) {
                        raise_status(status, ST_TIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                excl += static_cast<int64_t>(s & TS_VALUE);
                if (flag == TS_PREFIX) break;
                --i;
            }
            st_release_u64(&tile_state[tile], TS_PREFIX | static_cast<uint64_t>(excl + block_total));
        }
        s_excl = excl;
    }
    __syncthreads();
    int64_t run = s_excl + thread_excl;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        const int64_t idx = base + j;
        if (idx < m) out[idx] = run;
        run += v[j];
    }
    if (tile == (ntiles > 0 ? ntiles - 1 : 0) && threadIdx.x == 0) out[m] = s_excl + block_total;
}

// ---------------------------------------------------------------------------
// Write-combining scatter.
//
// Each round every thread holds V tuples.  Phase A: a shared atomicAdd on
// the partition's fill counter gives each tuple its position s in the
// partition's stream; s < W goes into the W-slot buffer.  Phase B: the tuple
// that took position W-1 flushes the full buffer as one aligned group;
// tuples with W <= s < Q (Q = fill rounded down to W: groups completed
// entirely inside this round) are stored straight to global memory.
// Phase C: the remaining tuples (s >= Q) refill the emptied buffer and the
// flusher moves the partition cursor by Q.  Every tuple is placed in the
// round it is read, whatever the skew.
template <typename K, int W>
struct WcTraits {
    static constexpr int TW = TupleTraits<K>::WORDS;
    static constexpr int BW = W * TW;  // words per buffer
    static_assert((BW * 4) % 16 == 0, "a buffer must be whole 16-byte vectors");
};

template <typename K>
__device__ __forceinline__ void tuple_words(uint32_t (&w)[TupleTraits<K>::WORDS], K key, int32_t row);

template <>
__device__ __forceinline__ void tuple_words<int32_t>(uint32_t (&w)[2], int32_t key, int32_t row)
{
    w[0] = hash_key(key);  // stored hash: the join compares and places by it
    w[1] = static_cast<uint32_t>(row);
}

template <>
__device__ __forceinline__ void tuple_words<int64_t>(uint32_t (&w)[4], int64_t key, int32_t row)
{
    const uint64_t u = static_cast<uint64_t>(key);
    w[0] = static_cast<uint32_t>(u);
    w[1] = static_cast<uint32_t>(u >> 32);
    w[2] = hash_key(key);  // stored hash: digits, buckets and fingerprints come from it
    w[3] = static_cast<uint32_t>(row);
}

template <int TW>
__device__ __forceinline__ void store_words(uint32_t* dst, const uint32_t (&w)[TW])
{
    if constexpr (TW == 2) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[1]);
    } else if constexpr (TW == 4) {
        *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
#pragma unroll
        for (int i = 0; i < TW; ++i) dst[i] = w[i];
    }
}

// One 32-byte store per sector: sm_100's 256-bit st.global makes every
// flushed sector a single L2 write request (two 16-byte stores of one
// sector are two requests, which bounds the scatter at the L2 request rate).
__device__ __forceinline__ void st_global_v8(uint32_t* g, const uint4& a, const uint4& b)
{
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(g), "r"(a.x), "r"(a.y), "r"(a.z),
                 "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
                 : "memory");
}

template <typename K, int W>
__device__ __forceinline__ void wc_flush(const uint32_t* sbuf, uint32_t* gdst)
{
    constexpr int BW = WcTraits<K, W>::BW;
    if constexpr ((BW * 4) % 32 == 0) {
#pragma unroll
        for (int q = 0; q < BW / 8; ++q)
            st_global_v8(gdst + 8 * q, reinterpret_cast<const uint4*>(sbuf)[2 * q],
                         reinterpret_cast<const uint4*>(sbuf)[2 * q + 1]);
    } else {
#pragma unroll
        for (int q = 0; q < BW / 4; ++q)
            reinterpret_cast<uint4*>(gdst)[q] = reinterpret_cast<const uint4*>(sbuf)[q];
    }
}



// Per-partition fill counts and output cursors of the write-combining
// scatter: two 4-byte arrays after the buffers.
struct WcState {
    int* fill;
    int* cur;
    __device__ static WcState at(uint32_t* after_buffers, int P)
    {
        int* f = reinterpret_cast<int*>(after_buffers);
        return WcState{f, f + P};
    }
    __device__ void init(int p, int cursor) const
    {
        fill[p] = 0;
        cur[p] = cursor;
    }
};

// One round of the write-combining scatter: every thread places its V
// tuples (words w, partition dv, ok = real) through the per-partition
// buffers of cap tuples (a multiple of the group size W).  Phase A: a shared
// atomic gives each tuple its slot in its partition's stream; slots below
// cap go to the buffer.  Phase B: the tuple in the last slot of each
// complete group inside the buffer flushes that group (one 32-byte store per
// sector); tuples of complete groups past the buffer go straight out.
// Phase C: the partial group after the last complete one moves to the
// buffer's front and the holder of the last complete slot advances the
// partition's cursor.  At every round's start a buffer holds fewer than W
// tuples.  Every thread of the CTA calls it (three barriers).
template <typename K, int W, int V>
__device__ __forceinline__ void wc_place(const uint32_t (&w)[V][TupleTraits<K>::WORDS], const uint32_t (&dv)[V],
                                         const bool (&ok)[V], uint32_t* buf, int cap, WcState fc,
                                         uint32_t* __restrict__ out, uint32_t out_cap, uint32_t* __restrict__ status)
{
    constexpr int TW = WcTraits<K, W>::TW;
    const int capw = cap * TW;
    int s[V], F[V], Q[V];
    // phase A
#pragma unroll
    for (int v = 0; v < V; ++v) {
        s[v] = ok[v] ? atomicAdd(&fc.fill[dv[v]], 1) : -1;
        if (ok[v] && s[v] < cap) store_words<TW>(buf + dv[v] * capw + s[v] * TW, w[v]);
    }
    __syncthreads();
    // phase B: only the tuples at or past the first group's last slot act
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (s[v] >= W - 1) {
            F[v] = fc.fill[dv[v]];
            Q[v] = F[v] & ~(W - 1);
            const uint32_t cur_p = static_cast<uint32_t>(fc.cur[dv[v]]);
            if (s[v] < cap) {
                if ((s[v] & (W - 1)) == W - 1) {
                    const int g0 = s[v] - (W - 1);  // first slot of the complete group
                    const uint32_t pos = cur_p + static_cast<uint32_t>(g0);
                    if (pos + static_cast<uint32_t>(W) <= out_cap)
                        wc_flush<K, W>(buf + dv[v] * capw + g0 * TW, out + static_cast<size_t>(pos) * TW);
                    else
                        raise_status(status, ST_INTERNAL);
                }
            } else if (s[v] < Q[v]) {
                const uint32_t pos = cur_p + static_cast<uint32_t>(s[v]);
                if (pos < out_cap)
                    store_words<TW>(out + static_cast<size_t>(pos) * TW, w[v]);
                else
                    raise_status(status, ST_INTERNAL);
            }
        }
    }
    __syncthreads();
    // phase C: a slot past the first group exists only where a group
    // completed (Q >= W), and then every slot from Q on was taken this round
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (s[v] >= W - 1 && Q[v] >= W) {
            if (s[v] >= Q[v]) store_words<TW>(buf + dv[v] * capw + (s[v] - Q[v]) * TW, w[v]);
            if (s[v] == Q[v] - 1) {
                fc.fill[dv[v]] = F[v] - Q[v];
                fc.cur[dv[v]] += Q[v];
            }
        }
    }
    __syncthreads();
}

// End of an item: pad every partial buffer to W tuples, write it, and check
// that each partition's cursor reached the end of its segment
// [offsets[p * n_items + item], offsets[p * n_items + item + 1]).
template <typename K, int W>
__device__ __forceinline__ void wc_finish(int P, uint32_t* buf, int cap, WcState fc, uint32_t* __restrict__ out,
                                          uint32_t out_cap,
                                          const int64_t* __restrict__ offsets, int32_t n_items, int32_t item,
                                          uint32_t* __restrict__ status)
{
    constexpr int TW = WcTraits<K, W>::TW;
    // final flush: pad every partial group (fewer than W tuples, at the
    // buffer's front) to W tuples and write it
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int fl = fc.fill[p];
        uint32_t cur_p = static_cast<uint32_t>(fc.cur[p]);
        if (fl > 0) {
            uint32_t* bq = buf + static_cast<size_t>(p) * cap * TW;
            for (int q = fl; q < W; ++q) {
                uint32_t pad[TW];
#pragma unroll
                for (int i = 0; i < TW; ++i) pad[i] = 0u;
                pad[TW - 1] = static_cast<uint32_t>(PAD_ROW);
                store_words<TW>(bq + q * TW, pad);
            }
            if (cur_p + static_cast<uint32_t>(W) <= out_cap)
                wc_flush<K, W>(bq, out + static_cast<size_t>(cur_p) * TW);
            else
                raise_status(status, ST_INTERNAL);
            cur_p += W;
        }
        if (cur_p != static_cast<uint32_t>(offsets[static_cast<int64_t>(p) * n_items + item + 1]))
            raise_status(status, ST_INTERNAL);
    }
}

// Scatter of a raw key column (row = key index).  V keys per thread per
// round (whole 16-byte vectors), the next two rounds' vectors loaded while
// the current round is processed.  Per partition the CTA keeps a buffer of
// cap tuples (whole groups of W), a fill count and an output cursor.
template <typename K, int THREADS, int V, int W, bool HASHD, bool HEAVY>
__global__ void __launch_bounds__(THREADS, 1) scatter_keys_kernel(const K* __restrict__ keys, int64_t n,
                                                                  int64_t chunk, int32_t n_items, DigitFn f,
                                                                  int32_t P, int32_t cap,
                                                                  const int64_t* __restrict__ offsets,
                                                                  uint32_t* __restrict__ out, uint32_t out_cap,
                                                                  uint32_t* __restrict__ status,
                                                                  typename HeavyArg<HEAVY>::type hs, HeavyOut ho)
{
    constexpr int TW = WcTraits<K, W>::TW;
    constexpr int VN = Vec16<K>::N;
    constexpr int NV = V / VN;  // vectors per thread per round
    static_assert(V % VN == 0, "V must be whole vectors");
    constexpr int ROUND = THREADS * V;
    extern __shared__ __align__(128) uint8_t smem[];
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem);
    const WcState fc = WcState::at(buf + static_cast<size_t>(P) * cap * TW, P);
    HeavyTable heavy;
    if constexpr (HEAVY) {
        // after the buffers and counters, on a 16-byte boundary (slots are
        // read as 16-byte words)
        heavy.bind(smem + heavy_table_offset(P, cap * TW));
        heavy.build<K>(hs, ho.heavy_row);  // ends with a barrier
    }
    const int lane = threadIdx.x & 31;

    __shared__ unsigned long long s_hbase;  // heavy pairs of the items before this one
    __shared__ uint32_t s_hcur;             // heavy pairs of this item so far
    for (int32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        for (int p = threadIdx.x; p < P; p += THREADS)
            fc.init(p, static_cast<int>(offsets[static_cast<int64_t>(p) * n_items + item]));
        if constexpr (HEAVY) {
            if (threadIdx.x < 32) {
                unsigned long long sum = 0;
                for (int j = threadIdx.x; j < item; j += 32) sum += ho.item_count[j];
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
                if (threadIdx.x == 0) {
                    s_hbase = sum;
                    s_hcur = 0;
                }
            }
        }
        __syncthreads();
        int64_t lo = static_cast<int64_t>(item) * chunk;
        const int64_t hi = lo + chunk < n ? lo + chunk : n;
        if (lo > hi) lo = hi;
        const K* kp = keys + lo;
        const uint32_t len = static_cast<uint32_t>(hi - lo);
        const uint32_t row0 = static_cast<uint32_t>(lo);

        // element e of vector j of this thread in the round at offset b:
        //   b + (j * THREADS + threadIdx.x) * VN + e
        auto load_round = [&](uint32_t b, K (&dst)[NV][VN]) {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const uint32_t at = b + (static_cast<uint32_t>(j) * THREADS + threadIdx.x) * VN;
                if (at + VN <= len) {
                    load_vec16<K>(kp + at, dst[j]);
                } else {
#pragma unroll
                    for (int e = 0; e < VN; ++e) dst[j][e] = at + e < len ? kp[at + e] : K(0);
                }
            }
        };
        K nxt[NV][VN], nxt2[NV][VN];
        if (len > 0) load_round(0, nxt);
        if (ROUND < len) load_round(ROUND, nxt2);
        for (uint32_t b = 0; b < len; b += ROUND) {
            K cur[NV][VN];
#pragma unroll
            for (int j = 0; j < NV; ++j)
#pragma unroll
                for (int e = 0; e < VN; ++e) {
                    cur[j][e] = nxt[j][e];
                    nxt[j][e] = nxt2[j][e];
                }
            if (b + 2 * ROUND < len) load_round(b + 2 * ROUND, nxt2);
            const bool full = b + ROUND <= len;

            uint32_t w[V][TW];
            uint32_t dv[V];  // the tuple's partition
            bool ok[V];
#pragma unroll
            for (int j = 0; j < NV; ++j)
#pragma unroll
                for (int e = 0; e < VN; ++e) {
                    const int v = j * VN + e;
                    const uint32_t at = b + (static_cast<uint32_t>(j) * THREADS + threadIdx.x) * VN + e;
                    ok[v] = full || at < len;
                    const K k = cur[j][e];
                    tuple_words<K>(w[v], k, static_cast<int32_t>(row0 + at));
                    uint32_t d;
                    if constexpr (HASHD) {
                        const uint32_t h = sizeof(K) == 4 ? w[v][0] : w[v][TW - 2];
                        d = (h >> f.shift) & f.mask;
                    } else {
                        d = static_cast<uint32_t>(static_cast<uint64_t>(k) >> f.shift) & f.mask;
                    }
                    dv[v] = d;
                }
            if constexpr (HEAVY) {
                // heavy probe keys: out of the partitions, matched here
                int32_t hb[V];
                int c = 0;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    hb[v] = -1;
                    if (ok[v]) {
                        const HeavyHit e = heavy.find(static_cast<K>(cur[v / VN][v % VN]));
                        if (e.idx >= 0) {
                            ok[v] = false;
                            hb[v] = e.row;
                            c += hb[v] >= 0 ? 1 : 0;
                        }
                    }
                }
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int tot = __shfl_sync(0xffffffffu, incl, 31);
                if (tot > 0) {
                    uint32_t base = 0;
                    if (lane == 31) base = atomicAdd(&s_hcur, static_cast<uint32_t>(tot));
                    base = __shfl_sync(0xffffffffu, base, 31);
                    if (ho.out_build) {
                        long long pos = static_cast<long long>(s_hbase) + base + (incl - c);
#pragma unroll
                        for (int v = 0; v < V; ++v) {
                            if (hb[v] >= 0) {
                                if (pos < ho.capacity) {
                                    ho.out_build[pos] = hb[v];
                                    ho.out_probe[pos] = static_cast<int32_t>(w[v][TW - 1]);
                                } else {
                                    raise_status(status, ST_CAPACITY);
                                }
                                ++pos;
                            }
                        }
                    }
                }
            }
            wc_place<K, W, V>(w, dv, ok, buf, cap, fc, out, out_cap, status);
        }
        wc_finish<K, W>(P, buf, cap, fc, out, out_cap, offsets, n_items, item, status);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Second radix pass (two-pass plans): the tuples of each pass-one partition
// are partitioned again by the next hash bits -- the reference's
// histogram_pass_two / partition_pass_two (partition_kernels.cuh:329-563),
// reading pass-one tuples instead of rewriting the input columns.
// Item (p1, c) is the c-th of C slices of pass-one partition p1's tuples
// [in_off[p1 * in_items], in_off[(p1 + 1) * in_items]); its tuples of sub-
// partition p2 go to the segment [off[p2 * n_items + item], ...).  With
// item = p1 * C + c that index is (p2 * P1 + p1) * C + c, so the join sees
// partition q = p2 * P1 + p1 as one range over C segments.
struct Pass2Items {
    const int64_t* in_off;  // pass-one segment offsets
    int32_t in_items;       // pass-one items
    int32_t C;              // slices per pass-one partition
};

__device__ __forceinline__ void pass2_range(const Pass2Items& it, int item, int64_t& lo, int64_t& hi)
{
    const int p1 = item / it.C, c = item % it.C;
    const int64_t start = it.in_off[static_cast<int64_t>(p1) * it.in_items];
    const int64_t end = it.in_off[static_cast<int64_t>(p1 + 1) * it.in_items];
    const int64_t per = (((end - start) + it.C - 1) / it.C + 15) & ~int64_t(15);
    lo = start + c * per;
    hi = lo + per < end ? lo + per : end;
    if (lo > hi) lo = hi;
}

// tuple i's words and whether it is a real (not padding) tuple
template <typename K>
__device__ __forceinline__ bool load_tuple_words(const uint32_t* __restrict__ t, int64_t i,
                                                 uint32_t (&w)[TupleTraits<K>::WORDS])
{
    if constexpr (TupleTraits<K>::WORDS == 2) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(t) + i);
        w[0] = v.x;
        w[1] = v.y;
    } else {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(t) + i);
        w[0] = v.x;
        w[1] = v.y;
        w[2] = v.z;
        w[3] = v.w;
    }
    return static_cast<int32_t>(w[TupleTraits<K>::WORDS - 1]) != PAD_ROW;
}

// the stored hash of a tuple (word 0 for 4-byte keys, word 2 for 8-byte keys)
template <typename K>
__device__ __forceinline__ uint32_t tuple_hash(const uint32_t (&w)[TupleTraits<K>::WORDS])
{
    return TupleTraits<K>::WORDS == 2 ? w[0] : w[TupleTraits<K>::WORDS - 2];
}

// Pass-two histogram: counts_T[p2 * n_items + item] and totals[p2 * P1 + p1]
// (zeroed by the caller).  Grid = n_items * hsplit CTAs.
template <typename K>
__global__ void __launch_bounds__(HIST_THREADS) hist_tuples_kernel(const uint32_t* __restrict__ tuples, Pass2Items it,
                                                                   int32_t n_items, int32_t hsplit, DigitFn f,
                                                                   int32_t P2, int32_t P1,
                                                                   uint32_t* __restrict__ counts_T,
                                                                   int32_t* __restrict__ totals)
{
    constexpr int TW = TupleTraits<K>::WORDS;
    extern __shared__ __align__(16) uint32_t cnt[];
    const int item = blockIdx.x / hsplit, part = blockIdx.x % hsplit;
    for (int p = threadIdx.x; p < P2; p += HIST_THREADS) cnt[p] = 0;
    __syncthreads();
    int64_t lo, hi;
    pass2_range(it, item, lo, hi);
    const int64_t per = (((hi - lo) + hsplit - 1) / hsplit + 15) & ~int64_t(15);
    int64_t s_lo = lo + part * per;
    const int64_t s_hi = s_lo + per < hi ? s_lo + per : hi;
    if (s_lo > s_hi) s_lo = s_hi;
    for (int64_t i = s_lo + threadIdx.x; i < s_hi; i += HIST_THREADS) {
        uint32_t w[TW];
        if (load_tuple_words<K>(tuples, i, w)) atomicAdd(&cnt[(tuple_hash<K>(w) >> f.shift) & f.mask], 1u);
    }
    __syncthreads();
    const int p1 = item / it.C;
    for (int p = threadIdx.x; p < P2; p += HIST_THREADS) {
        const uint32_t c = cnt[p];
        if (c) {
            atomicAdd(&counts_T[static_cast<int64_t>(p) * n_items + item], c);
            atomicAdd(&totals[static_cast<int64_t>(p) * P1 + p1], static_cast<int32_t>(c));
        }
    }
}

// Pass-two scatter: the pass-one tuples of each item, placed by the next
// hash bits through the same write-combining buffers as the first pass.
// VT tuples per thread per round, the next round's loaded ahead.
template <typename K, int THREADS, int VT, int W>
__global__ void __launch_bounds__(THREADS, 1) scatter_tuples_kernel(const uint32_t* __restrict__ in, Pass2Items it,
                                                                    int32_t n_items, DigitFn f, int32_t P,
                                                                    int32_t cap, const int64_t* __restrict__ offsets,
                                                                    uint32_t* __restrict__ out, uint32_t out_cap,
                                                                    uint32_t* __restrict__ status)
{
    constexpr int TW = WcTraits<K, W>::TW;
    constexpr int ROUND = THREADS * VT;
    extern __shared__ __align__(128) uint8_t smem[];
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem);
    const WcState fc = WcState::at(buf + static_cast<size_t>(P) * cap * TW, P);
    for (int32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        for (int p = threadIdx.x; p < P; p += THREADS)
            fc.init(p, static_cast<int>(offsets[static_cast<int64_t>(p) * n_items + item]));
        __syncthreads();
        int64_t lo, hi;
        pass2_range(it, item, lo, hi);
        uint32_t nw[VT][TW];
        bool nok[VT];
        auto load_round = [&](int64_t b) {
#pragma unroll
            for (int v = 0; v < VT; ++v) {
                const int64_t i = b + static_cast<int64_t>(v) * THREADS + threadIdx.x;
                nok[v] = i < hi && load_tuple_words<K>(in, i, nw[v]);
            }
        };
        if (lo < hi) load_round(lo);
        for (int64_t b = lo; b < hi; b += ROUND) {
            uint32_t w[VT][TW];
            uint32_t dv[VT];
            bool ok[VT];
#pragma unroll
            for (int v = 0; v < VT; ++v) {
                ok[v] = nok[v];
#pragma unroll
                for (int i = 0; i < TW; ++i) w[v][i] = nw[v][i];
                dv[v] = (tuple_hash<K>(w[v]) >> f.shift) & f.mask;
            }
            if (b + ROUND < hi) load_round(b + ROUND);
            wc_place<K, W, VT>(w, dv, ok, buf, cap, fc, out, out_cap, status);
        }
        wc_finish<K, W>(P, buf, cap, fc, out, out_cap, offsets, n_items, item, status);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Batches of joins: histogram and scatter over the items (SegItem) of many
// join sides in one launch each.

// Histogram of the items (grid = items * hsplit, hsplit CTAs per item).
template <typename K>
__global__ void __launch_bounds__(HIST_THREADS) hist_seg_kernel(const SegItem* __restrict__ items, int32_t hsplit,
                                                                uint32_t* __restrict__ counts,
                                                                int32_t* __restrict__ totals)
{
    extern __shared__ __align__(16) uint32_t cnt[];
    const SegItem it = items[blockIdx.x / hsplit];
    const int part = blockIdx.x % hsplit;
    for (int p = threadIdx.x; p < it.P; p += HIST_THREADS) cnt[p] = 0;
    __syncthreads();
    const K* keys = static_cast<const K*>(it.keys);
    const int64_t per = (((it.hi - it.lo) + hsplit - 1) / hsplit + 15) & ~int64_t(15);
    int64_t s_lo = it.lo + part * per;
    const int64_t s_hi = s_lo + per < it.hi ? s_lo + per : it.hi;
    if (s_lo > s_hi) s_lo = s_hi;
    // SEG_UNROLL independent loads in flight per thread, then their counts
    constexpr int SEG_UNROLL = 8;
    int64_t i = s_lo + threadIdx.x;
    for (; i + (SEG_UNROLL - 1) * HIST_THREADS < s_hi; i += SEG_UNROLL * HIST_THREADS) {
        K k[SEG_UNROLL];
#pragma unroll
        for (int u = 0; u < SEG_UNROLL; ++u) k[u] = __ldg(keys + i + u * HIST_THREADS);
#pragma unroll
        for (int u = 0; u < SEG_UNROLL; ++u) atomicAdd(&cnt[(hash_key(k[u]) >> it.f.shift) & it.f.mask], 1u);
    }
    for (; i < s_hi; i += HIST_THREADS) atomicAdd(&cnt[(hash_key(keys[i]) >> it.f.shift) & it.f.mask], 1u);
    __syncthreads();
    for (int p = threadIdx.x; p < it.P; p += HIST_THREADS) {
        const uint32_t c = cnt[p];
        if (c) {
            atomicAdd(&counts[it.cnt_base + static_cast<int64_t>(p) * it.seg_items + it.item], c);
            atomicAdd(&totals[it.tot_base + p], static_cast<int32_t>(c));
        }
    }
}

// Write-combining scatter of the items (persistent grid; buffers sized for
// the largest partition count of the batch, Pmax).
template <typename K, int THREADS, int VT, int W>
__global__ void __launch_bounds__(THREADS, 1) scatter_seg_kernel(const SegItem* __restrict__ items, int32_t n_items,
                                                                 int32_t Pmax, int32_t cap,
                                                                 const int64_t* __restrict__ offsets,
                                                                 uint32_t* __restrict__ out, uint32_t out_cap,
                                                                 uint32_t* __restrict__ status)
{
    constexpr int TW = WcTraits<K, W>::TW;
    constexpr int ROUND = THREADS * VT;
    extern __shared__ __align__(128) uint8_t smem[];
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem);
    const WcState fc = WcState::at(buf + static_cast<size_t>(Pmax) * cap * TW, Pmax);
    for (int32_t i = blockIdx.x; i < n_items; i += gridDim.x) {
        const SegItem it = items[i];
        const int64_t* off = offsets + it.cnt_base;
        for (int p = threadIdx.x; p < it.P; p += THREADS)
            fc.init(p, static_cast<int>(off[static_cast<int64_t>(p) * it.seg_items + it.item]));
        __syncthreads();
        const K* keys = static_cast<const K*>(it.keys);
        K nk[VT];
        auto load_round = [&](int64_t b) {
#pragma unroll
            for (int v = 0; v < VT; ++v) {
                const int64_t r = b + static_cast<int64_t>(v) * THREADS + threadIdx.x;
                nk[v] = r < it.hi ? keys[r] : K(0);
            }
        };
        if (it.lo < it.hi) load_round(it.lo);
        for (int64_t b = it.lo; b < it.hi; b += ROUND) {
            uint32_t w[VT][TW];
            uint32_t dv[VT];
            bool ok[VT];
#pragma unroll
            for (int v = 0; v < VT; ++v) {
                const int64_t r = b + static_cast<int64_t>(v) * THREADS + threadIdx.x;
                ok[v] = r < it.hi;
                tuple_words<K>(w[v], nk[v], static_cast<int32_t>(r));
                dv[v] = (tuple_hash<K>(w[v]) >> it.f.shift) & it.f.mask;
            }
            if (b + ROUND < it.hi) load_round(b + ROUND);
            wc_place<K, W, VT>(w, dv, ok, buf, cap, fc, out, out_cap, status);
        }
        wc_finish<K, W>(it.P, buf, cap, fc, out, out_cap, off, it.seg_items, it.item, status);
        __syncthreads();
    }
}

}  // namespace pj
