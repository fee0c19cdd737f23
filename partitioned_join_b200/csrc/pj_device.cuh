// pj_device.cuh -- device building blocks shared by every kernel:
// the reference's hash, digit and slot functions, the partitioned tuple
// layout, and bounded-wait helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pj {

// ---------------------------------------------------------------------------
// Device status word (in the workspace).  Kernels OR bits in; pj_check()
// reads and clears it.
enum : uint32_t {
    ST_CAPACITY = 1u << 0,  // more matches than output capacity
    ST_OVERFLOW = 1u << 1,  // a shared-memory table ran out of slots
    ST_TIMEOUT = 1u << 2,   // a bounded spin gave up
    ST_INTERNAL = 1u << 3,  // a consistency check failed (e.g. scatter overran its segment)
};

__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bit)
{
    atomicOr(status, bit);
}

// ---------------------------------------------------------------------------
// MurmurHash3_x86_32 with seed 0 over the key's little-endian bytes, equal
// bit for bit to MurmurHash3_32<K>::operator() (hash_functions.cuh:80-119).
// Written from the published algorithm (Appleby, smhasher); the rotations
// use the funnel shifter.
__device__ __forceinline__ uint32_t mm_block(uint32_t h, uint32_t k)
{
    k *= 0xcc9e2d51u;
    k = __funnelshift_l(k, k, 15);
    k *= 0x1b873593u;
    h ^= k;
    h = __funnelshift_l(h, h, 13);
    return h * 5u + 0xe6546b64u;
}

__device__ __forceinline__ uint32_t mm_fmix(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ uint32_t hash_key(int32_t k)
{
    return mm_fmix(mm_block(0u, static_cast<uint32_t>(k)) ^ 4u);
}

__device__ __forceinline__ uint32_t hash_key(int64_t k)
{
    const uint64_t u = static_cast<uint64_t>(k);
    uint32_t h = mm_block(0u, static_cast<uint32_t>(u));
    h = mm_block(h, static_cast<uint32_t>(u >> 32));
    return mm_fmix(h ^ 8u);
}

// ---------------------------------------------------------------------------
// Partition digit.  RAW: (key >> shift) & mask -- the reference's
// ((P1-1) << b2 & key) >> b2 and key & (P2-1) (partition_kernels.cuh:168,380)
// are this with shift = b2 and shift = 0.  HASH: (h >> shift) & mask with
// the digit taken from the top hash bits.
struct DigitFn {
    int32_t mode;   // PJ_DIGIT_RAW = 0, PJ_DIGIT_HASH = 1
    int32_t shift;
    uint32_t mask;  // 2^bits - 1 (0: a single partition)
};

template <typename K>
__device__ __forceinline__ uint32_t digit_of(const DigitFn& f, K key, uint32_t h)
{
    const uint32_t src = f.mode == 1 ? (f.mask ? (h >> f.shift) : 0u)
                                     : static_cast<uint32_t>(static_cast<uint64_t>(key) >> f.shift);
    return src & f.mask;
}

// ---------------------------------------------------------------------------
// Slot inside a partition table of T slots.
//   FAST: the hash bits not used by digits (skip) or slices (sbits), left
//         aligned, mapped to [0, T) by a multiply-high (Lemire's range
//         reduction).
//   REF:  abs((int)h % T) -- hash_join_kernels.cuh:100-101 with int_fastdiv's
//         truncating signed remainder (int_fastdiv.h:118-133).
__device__ __forceinline__ uint32_t slot_fast(uint32_t h, int skip, uint32_t T)
{
    return __umulhi(h << skip, T);
}

__device__ __forceinline__ uint32_t slot_ref(uint32_t h, int32_t T)
{
    const int32_t r = static_cast<int32_t>(h) % T;
    return static_cast<uint32_t>(r < 0 ? -r : r);
}

// ---------------------------------------------------------------------------
// Partitioned tuples.  4-byte keys: {murmur(key), row} (8 B).  8-byte keys:
// {key_lo, key_hi, murmur(key), row} (16 B: one aligned vector, and the join
// never hashes again).  The row is the last word; padding tuples have
// row == -1.
template <typename K> struct TupleTraits;
template <> struct TupleTraits<int32_t> { static constexpr int WORDS = 2; };
template <> struct TupleTraits<int64_t> { static constexpr int WORDS = 4; };

constexpr int32_t PAD_ROW = -1;

// ---------------------------------------------------------------------------
// Exclusive scan, in place, of the 16-bit counts packed two per word in
// w[0 .. nwords).  Totals stay below 65536.  Ends with __syncthreads().
template <int THREADS>
__device__ __forceinline__ void scan_u16_pairs(uint32_t* w, int nwords, uint32_t* s_warp)
{
    // an odd run length: the lanes of a warp then walk 32 different banks
    const int per = ((nwords + THREADS - 1) / THREADS) | 1;
    const int a = threadIdx.x * per;
    const int b = a + per < nwords ? a + per : nwords;
    uint32_t sum = 0;
    for (int i = a; i < b; ++i) {
        const uint32_t x = w[i];
        sum += (x & 0xffffu) + (x >> 16);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t x = lane < THREADS / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < THREADS / 32) s_warp[lane] = x;
    }
    __syncthreads();
    uint32_t run = incl - sum + (warp > 0 ? s_warp[warp - 1] : 0u);
    for (int i = a; i < b; ++i) {
        const uint32_t x = w[i];
        const uint32_t c0 = x & 0xffffu, c1 = x >> 16;
        w[i] = (run & 0xffffu) | ((run + c0) << 16);
        run += c0 + c1;
    }
    __syncthreads();
}

// Bounded spin: iterations before a wait gives up and raises ST_TIMEOUT.
constexpr uint32_t SPIN_LIMIT = 1u << 24;

}  // namespace pj
