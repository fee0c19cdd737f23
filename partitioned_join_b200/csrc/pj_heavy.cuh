// pj_heavy.cuh -- the heavy-key path: probe keys that occur very often
// (Zipf-skewed probe sides) bypass partitioning and are matched at once
// against a small table that every CTA holds (broadcast probe).
//
// Reference counterpart: skewed_data_handler.cuh:21-91 detects oversized
// partitions after partitioning and splits their work over more CTAs; every
// heavy probe row is still partitioned, scattered and probed.  Here the
// planner names up to MAX_HEAVY heavy probe keys from a sample of the probe
// column, and then (unique build keys only):
//   1. heavy_rows_kernel finds the build row of each heavy key (one read of
//      the build keys);
//   2. the probe side's histogram skips heavy keys and counts, per item, the
//      heavy rows that have a build row; its scatter writes (heavy_row,
//      probe_row) straight to the output instead of partitioning the tuple --
//      item i's pairs at exact positions after those of items < i, inside
//      [0, H) of the output;
//   3. the join kernel reserves its output chunks after H, and the output
//      fix-up counts H in.
// A heavy key without a build row drops its probe rows (no match).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_device.cuh"

namespace pj {

constexpr int MAX_HEAVY = 256;    // = PJ_MAX_HEAVY
constexpr int HEAVY_SLOTS = 512;  // open-addressing slots of a CTA's heavy table

// Heavy keys, passed by value as a kernel parameter (graph-capturable).
struct HeavySet {
    int32_t n;
    int32_t pad;
    int64_t keys[MAX_HEAVY];
};
struct NoHeavy {};
template <bool HEAVY> struct HeavyArg { using type = NoHeavy; };
template <> struct HeavyArg<true> { using type = HeavySet; };

// Home slot of a key in a heavy table: a multiplicative hash of the key
// (the top bits of key * 2^64/phi; Knuth, TAOCP vol. 3, 6.4) -- a few
// instructions where the histogram would otherwise need a murmur hash.
template <typename K>
__device__ __forceinline__ uint32_t heavy_slot_of(K k)
{
    return static_cast<uint32_t>((static_cast<uint64_t>(static_cast<int64_t>(k)) * 0x9e3779b97f4a7c15ull) >> 55);
}
static_assert(HEAVY_SLOTS == 512, "heavy_slot_of keeps 9 bits");

// Result of a heavy-table lookup.
struct HeavyHit {
    int32_t idx;  // index in the heavy set, -1: not a heavy key
    int32_t row;  // its build row, -1: none
};

// A CTA's copy of the heavy set in shared memory: home slot heavy_slot_of,
// linear probing.  A slot is one 16-byte word {key, index, build row}
// (index -1: empty), so a lookup is one shared load per probe.
struct HeavyTable {
    struct Slot {
        int64_t key;
        int32_t idx;
        int32_t row;
    };
    static constexpr size_t BYTES = HEAVY_SLOTS * sizeof(Slot);
    Slot* slot;

    __device__ void bind(uint8_t* smem) { slot = reinterpret_cast<Slot*>(smem); }
    // every thread of the CTA; ends with a barrier.  heavy_row: build rows of
    // the heavy keys (nullptr: not known yet)
    template <typename K>
    __device__ void build(const HeavySet& hs, const int32_t* __restrict__ heavy_row)
    {
        int32_t* idx_word = reinterpret_cast<int32_t*>(slot);
        for (int s = threadIdx.x; s < HEAVY_SLOTS; s += blockDim.x) slot[s] = Slot{0, -1, -1};
        __syncthreads();
        for (int t = threadIdx.x; t < hs.n; t += blockDim.x) {
            const K k = static_cast<K>(hs.keys[t]);
            uint32_t s = heavy_slot_of(k);
            for (int tries = 0; tries < HEAVY_SLOTS; ++tries) {
                if (atomicCAS(&idx_word[4 * s + 2], -1, t) == -1) {
                    slot[s].key = static_cast<int64_t>(k);
                    slot[s].row = heavy_row ? heavy_row[t] : -1;
                    break;
                }
                s = (s + 1) & (HEAVY_SLOTS - 1);
            }
        }
        __syncthreads();
    }
    // lookup of key k.  The home slot answers almost every lookup (the table
    // is at most half full); collisions walk on.
    template <typename K>
    __device__ __forceinline__ HeavyHit find(K k) const
    {
        const uint64_t want = static_cast<uint64_t>(static_cast<int64_t>(k));
        uint32_t s = heavy_slot_of(k);
        for (int tries = 0; tries < HEAVY_SLOTS; ++tries) {
            const int4 v = *reinterpret_cast<const int4*>(&slot[s]);
            if (v.z < 0) break;
            if ((static_cast<uint64_t>(static_cast<uint32_t>(v.y)) << 32 | static_cast<uint32_t>(v.x)) == want)
                return HeavyHit{v.z, v.w};
            s = (s + 1) & (HEAVY_SLOTS - 1);
        }
        return HeavyHit{-1, -1};
    }
};

// heavy_row[i] = the build row holding heavy key i (unique build keys; the
// caller sets heavy_row to -1 first).
template <typename K>
__global__ void __launch_bounds__(512) heavy_rows_kernel(const K* __restrict__ keys, int64_t n, HeavySet hs,
                                                         int32_t* __restrict__ heavy_row)
{
    __shared__ __align__(16) uint8_t smem[HeavyTable::BYTES];
    HeavyTable t;
    t.bind(smem);
    t.build<K>(hs, nullptr);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const HeavyHit e = t.find(keys[i]);
        if (e.idx >= 0) heavy_row[e.idx] = static_cast<int32_t>(i);
    }
}

// Position of sample s in a column of n rows (SplitMix64 of s).
__device__ __forceinline__ int64_t sample_pos(int s, int64_t n)
{
    uint64_t x = static_cast<uint64_t>(s) * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    x ^= x >> 31;
    return static_cast<int64_t>(x % static_cast<uint64_t>(n));
}

// Keys at pseudo-random positions of a column (the planner's sample).
template <typename K>
__global__ void sample_keys_kernel(const K* __restrict__ keys, int64_t n, int32_t samples, int64_t* __restrict__ out)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < samples; s += gridDim.x * blockDim.x)
        out[s] = static_cast<int64_t>(keys[sample_pos(s, n)]);
}

// H = the heavy pairs of every item: the output count so far, where the
// join's output chunks begin.  One warp.
static __global__ void heavy_total_kernel(const unsigned long long* __restrict__ item_count, int32_t n_items,
                                   unsigned long long* __restrict__ total, unsigned long long* __restrict__ count)
{
    unsigned long long sum = 0;
    for (int j = threadIdx.x; j < n_items; j += 32) sum += item_count[j];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if (threadIdx.x == 0) {
        *total = sum;
        *count = sum;
    }
}

}  // namespace pj
