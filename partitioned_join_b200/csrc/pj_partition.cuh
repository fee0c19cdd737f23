// pj_partition.cuh -- radix histogram, decoupled look-back scan and
// write-combining scatter.
//
// Layout of one partitioned column.  The input is cut into n_items equal
// chunks ("items", one per resident scatter CTA).  Item i's tuples of
// partition p form the segment [off[p*n_items + i], off[p*n_items + i + 1])
// of the output, where off is the exclusive scan of the per-(p, i) counts,
// each rounded up to W tuples.  So partitions are contiguous
// (partition p = [off[p*n_items], off[(p+1)*n_items]) ), every segment starts
// on a W-tuple boundary (one or more whole 32-byte sectors), and the padding
// tuples that fill a segment's last W-group carry row = -1.
//
// Reference counterparts: histogram_pass_one (partition_kernels.cuh:141-194),
// the ExclusiveSum + copy of partitioned_join.cuh:86-88, partition_pass_one
// (partition_kernels.cuh:197-326).  The reference stages an 8 192-key tile in
// shared memory and flushes each partition's run with 32 threads; here each
// CTA keeps a W-tuple write-combining buffer per partition and only ever
// writes whole aligned sectors, so the DRAM sees full-sector writes at any
// fan-out.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_bulk.cuh"
#include "pj_device.cuh"

namespace pj {

constexpr int HIST_THREADS = 1024;
constexpr int HIST_V = 4;       // keys per thread per round
constexpr int HIST_NSTAGE = 3;

template <typename K>
__device__ __forceinline__ uint32_t key_digit(const DigitFn& f, K key)
{
    return digit_of(f, key, f.mode == 1 ? hash_key(key) : 0u);
}

// Per-(partition, item) histogram of one key column.  counts_T[p*n_items+i]
// (p-major, the order the scan wants) and, if totals != nullptr,
// atomicAdd of every partition's count into totals[p].
template <typename K>
__global__ void __launch_bounds__(HIST_THREADS) hist_keys_kernel(const K* __restrict__ keys, int64_t n,
                                                                 int64_t chunk, int32_t n_items, DigitFn f,
                                                                 int32_t P, uint32_t* __restrict__ counts_T,
                                                                 int32_t* __restrict__ totals,
                                                                 uint32_t* __restrict__ status)
{
    constexpr int ROUND = HIST_THREADS * HIST_V;
    constexpr int STAGE_BYTES = ROUND * static_cast<int>(sizeof(K));
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* stages = smem;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(smem + HIST_NSTAGE * STAGE_BYTES);
    __shared__ uint64_t bars[HIST_NSTAGE];

    BulkRing<HIST_NSTAGE, STAGE_BYTES> ring;
    ring.stages = stages;
    ring.bars = bars;
    ring.phase_bits = 0;
    ring.init_barriers();

    for (int32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        for (int p = threadIdx.x; p < P; p += HIST_THREADS) cnt[p] = 0;
        __syncthreads();
        int64_t lo = static_cast<int64_t>(item) * chunk;
        int64_t hi = lo + chunk < n ? lo + chunk : n;
        if (lo > hi) lo = hi;
        const int64_t bulk_keys = (((hi - lo) * static_cast<int64_t>(sizeof(K))) & ~int64_t(15)) / sizeof(K);
        ring.start(keys + lo, bulk_keys * static_cast<int64_t>(sizeof(K)), status);
        const int64_t nch = ring.num_chunks();
        for (int64_t c = 0; c < nch; ++c) {
            const K* sk = reinterpret_cast<const K*>(ring.wait(c));
            const int64_t left = bulk_keys - c * ROUND;
            const int cntk = left < ROUND ? static_cast<int>(left) : ROUND;
#pragma unroll
            for (int v = 0; v < HIST_V; ++v) {
                const int j = v * HIST_THREADS + threadIdx.x;
                if (j < cntk) atomicAdd(&cnt[key_digit(f, sk[j])], 1u);
            }
            __syncthreads();
            ring.release(c);
        }
        for (int64_t j = lo + bulk_keys + threadIdx.x; j < hi; j += HIST_THREADS)
            atomicAdd(&cnt[key_digit(f, keys[j])], 1u);
        __syncthreads();
        for (int p = threadIdx.x; p < P; p += HIST_THREADS) {
            const uint32_t c = cnt[p];
            counts_T[static_cast<int64_t>(p) * n_items + item] = c;
            if (totals != nullptr && c) atomicAdd(&totals[p], static_cast<int32_t>(c));
        }
        __syncthreads();
    }
}

// Global digit histogram (no per-item split): the stage entry point
// pj_radix_histogram and the exact planner.  Grid-stride over the keys.
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

template <typename TIn>
__global__ void __launch_bounds__(SCAN_THREADS) lookback_scan_kernel(const TIn* __restrict__ in, int64_t m,
                                                                     uint32_t round_to, int64_t* __restrict__ out,
                                                                     uint64_t* __restrict__ tile_state,
                                                                     uint32_t* __restrict__ tile_counter,
                                                                     uint32_t* __restrict__ status)
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
    // block exclusive scan of the per-thread sums
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
    int64_t thread_excl = incl - sum + (warp > 0 ? s_warp[warp - 1] : 0);

    if (threadIdx.x == 0) {
        int64_t excl = 0;
        if (tile == 0) {
            st_release_u64(&tile_state[0], TS_PREFIX | static_cast<uint64_t>(block_total));
        } else {
            st_release_u64(&tile_state[tile], TS_AGG | static_cast<uint64_t>(block_total));
            int64_t i = tile - 1;
            uint32_t spins = 0;
            while (i >= 0) {
                const uint64_t s = ld_acquire_u64(&tile_state[i]);
                const uint64_t flag = s & ~TS_VALUE;
                if (flag == 0) {
                    if (++spins > SPIN_LIMIT) {
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
// that took position W-1 flushes the full buffer as whole sectors; tuples
// with W <= s < Q (Q = fill rounded down to W, i.e. sectors completed
// entirely inside this round) are stored straight to global memory.  Phase C:
// the remaining tuples (s >= Q) refill the emptied buffer; the flusher moves
// the partition cursor by Q.  Every tuple is placed in the round it is read,
// whatever the skew.
template <typename K, int W>
struct WcTraits {
    static constexpr int TW = TupleTraits<K>::WORDS;
    static constexpr int BW = W * TW;  // words per buffer
    static_assert((BW * 4) % 32 == 0, "a buffer must be whole 32-byte sectors");
};

template <typename K, int W, int V>
__device__ __forceinline__ void wc_phase_a(const K (&key)[V], const int32_t (&row)[V], const bool (&ok)[V],
                                           const uint32_t (&d)[V], int (&s)[V], uint32_t* buf, int* fill)
{
    constexpr int TW = WcTraits<K, W>::TW, BW = WcTraits<K, W>::BW;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (ok[v]) {
            s[v] = atomicAdd(&fill[d[v]], 1);
            if (s[v] < W) put_tuple_words<K>(buf + static_cast<size_t>(d[v]) * BW + s[v] * TW, key[v], row[v]);
        }
    }
}

template <typename K, int W>
__device__ __forceinline__ void wc_flush(const uint32_t* sbuf, uint32_t* gdst)
{
    constexpr int BW = WcTraits<K, W>::BW;
#pragma unroll
    for (int q = 0; q < BW / 4; ++q)
        reinterpret_cast<uint4*>(gdst)[q] = reinterpret_cast<const uint4*>(sbuf)[q];
}

template <typename K, int W, int V>
__device__ __forceinline__ void wc_phase_b(const K (&key)[V], const int32_t (&row)[V], const bool (&ok)[V],
                                           const uint32_t (&d)[V], const int (&s)[V], int (&F)[V], int (&Q)[V],
                                           const uint32_t* buf, const int* fill, const uint32_t* cursor,
                                           uint32_t* __restrict__ out, uint32_t out_cap, uint32_t* status)
{
    constexpr int TW = WcTraits<K, W>::TW, BW = WcTraits<K, W>::BW;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (ok[v]) {
            F[v] = fill[d[v]];
            Q[v] = F[v] - F[v] % W;
            const uint32_t cur = cursor[d[v]];
            if (s[v] == W - 1) {
                if (cur + static_cast<uint32_t>(W) <= out_cap)
                    wc_flush<K, W>(buf + static_cast<size_t>(d[v]) * BW, out + static_cast<size_t>(cur) * TW);
                else
                    raise_status(status, ST_INTERNAL);
            } else if (s[v] >= W && s[v] < Q[v]) {
                const uint32_t pos = cur + static_cast<uint32_t>(s[v]);
                if (pos < out_cap)
                    put_tuple_words<K>(out + static_cast<size_t>(pos) * TW, key[v], row[v]);
                else
                    raise_status(status, ST_INTERNAL);
            }
        }
    }
}

template <typename K, int W, int V>
__device__ __forceinline__ void wc_phase_c(const K (&key)[V], const int32_t (&row)[V], const bool (&ok)[V],
                                           const uint32_t (&d)[V], const int (&s)[V], const int (&F)[V],
                                           const int (&Q)[V], uint32_t* buf, int* fill, uint32_t* cursor)
{
    constexpr int TW = WcTraits<K, W>::TW, BW = WcTraits<K, W>::BW;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (ok[v]) {
            if (s[v] >= W && s[v] >= Q[v])
                put_tuple_words<K>(buf + static_cast<size_t>(d[v]) * BW + (s[v] - Q[v]) * TW, key[v], row[v]);
            if (s[v] == W - 1) {
                cursor[d[v]] += static_cast<uint32_t>(Q[v]);
                fill[d[v]] = F[v] - Q[v];
            }
        }
    }
}

template <typename K>
__device__ __forceinline__ void pad_tuple_words(uint32_t* dst)
{
    put_tuple_words<K>(dst, K(0), PAD_ROW);
}

// Shared memory of the scatter kernel: stages + buffers + fill + cursor.
template <typename K, int THREADS, int V, int W, int NSTAGE>
struct ScatterSmem {
    static constexpr int ROUND = THREADS * V;
    static constexpr int STAGE_BYTES = ROUND * static_cast<int>(sizeof(K));
    static size_t bytes(int P)
    {
        return static_cast<size_t>(NSTAGE) * STAGE_BYTES + static_cast<size_t>(P) * WcTraits<K, W>::BW * 4 +
               static_cast<size_t>(P) * 8;
    }
};

// Scatter of a raw key column (row = key index).
template <typename K, int THREADS, int V, int W, int NSTAGE>
__global__ void __launch_bounds__(THREADS, 1) scatter_keys_kernel(const K* __restrict__ keys, int64_t n,
                                                                  int64_t chunk, int32_t n_items, DigitFn f,
                                                                  int32_t P, const int64_t* __restrict__ offsets,
                                                                  uint32_t* __restrict__ out, uint32_t out_cap,
                                                                  uint32_t* __restrict__ status)
{
    using SM = ScatterSmem<K, THREADS, V, W, NSTAGE>;
    constexpr int TW = WcTraits<K, W>::TW, BW = WcTraits<K, W>::BW;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* stages = smem;
    uint32_t* buf = reinterpret_cast<uint32_t*>(smem + NSTAGE * SM::STAGE_BYTES);
    int* fill = reinterpret_cast<int*>(buf + static_cast<size_t>(P) * BW);
    uint32_t* cursor = reinterpret_cast<uint32_t*>(fill + P);
    __shared__ uint64_t bars[NSTAGE];

    BulkRing<NSTAGE, SM::STAGE_BYTES> ring;
    ring.stages = stages;
    ring.bars = bars;
    ring.phase_bits = 0;
    ring.init_barriers();

    for (int32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        for (int p = threadIdx.x; p < P; p += THREADS) {
            fill[p] = 0;
            cursor[p] = static_cast<uint32_t>(offsets[static_cast<int64_t>(p) * n_items + item]);
        }
        __syncthreads();
        int64_t lo = static_cast<int64_t>(item) * chunk;
        const int64_t hi = lo + chunk < n ? lo + chunk : n;
        if (lo > hi) lo = hi;
        const int64_t bulk_keys = (((hi - lo) * static_cast<int64_t>(sizeof(K))) & ~int64_t(15)) / sizeof(K);
        ring.start(keys + lo, bulk_keys * static_cast<int64_t>(sizeof(K)), status);
        const int64_t nch = ring.num_chunks();
        const int64_t tail_chunks = (hi - lo - bulk_keys) > 0 ? 1 : 0;
        for (int64_t c = 0; c < nch + tail_chunks; ++c) {
            K key[V];
            int32_t row[V];
            bool ok[V];
            uint32_t d[V];
            int s[V], F[V], Q[V];
            if (c < nch) {
                const K* sk = reinterpret_cast<const K*>(ring.wait(c));
                const int64_t cbase = lo + c * SM::ROUND;
                const int64_t left = bulk_keys - c * SM::ROUND;
                const int cnt = left < SM::ROUND ? static_cast<int>(left) : SM::ROUND;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = v * THREADS + threadIdx.x;
                    ok[v] = j < cnt;
                    key[v] = ok[v] ? sk[j] : K(0);
                    row[v] = static_cast<int32_t>(cbase + j);
                    d[v] = ok[v] ? key_digit(f, key[v]) : 0u;
                }
            } else {  // the < 16-byte tail the bulk copies leave out
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int64_t j = lo + bulk_keys + v * THREADS + threadIdx.x;
                    ok[v] = j < hi;
                    key[v] = ok[v] ? keys[j] : K(0);
                    row[v] = static_cast<int32_t>(j);
                    d[v] = ok[v] ? key_digit(f, key[v]) : 0u;
                }
            }
            wc_phase_a<K, W, V>(key, row, ok, d, s, buf, fill);
            __syncthreads();
            if (c < nch) ring.release(c);
            wc_phase_b<K, W, V>(key, row, ok, d, s, F, Q, buf, fill, cursor, out, out_cap, status);
            __syncthreads();
            wc_phase_c<K, W, V>(key, row, ok, d, s, F, Q, buf, fill, cursor);
            __syncthreads();
        }
        // final flush: pad every partial buffer to W tuples and write it
        for (int p = threadIdx.x; p < P; p += THREADS) {
            const int fl = fill[p];
            uint32_t cur = cursor[p];
            if (fl > 0) {
                uint32_t* b = buf + static_cast<size_t>(p) * BW;
                for (int q = fl; q < W; ++q) pad_tuple_words<K>(b + q * TW);
                if (cur + static_cast<uint32_t>(W) <= out_cap)
                    wc_flush<K, W>(b, out + static_cast<size_t>(cur) * TW);
                else
                    raise_status(status, ST_INTERNAL);
                cur += W;
            }
            if (cur != static_cast<uint32_t>(offsets[static_cast<int64_t>(p) * n_items + item + 1]))
                raise_status(status, ST_INTERNAL);
        }
        __syncthreads();
    }
}

}  // namespace pj
