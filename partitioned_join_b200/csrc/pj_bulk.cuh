// pj_bulk.cuh -- a staged streaming reader: one thread issues bulk
// asynchronous copies (cp.async.bulk, the TMA engine's untiled form) of
// consecutive byte ranges of a global array into a ring of shared-memory
// stages, each guarded by an mbarrier; all threads of the CTA consume the
// stages in order.  Every wait is bounded.
//
// Requirements (checked by the callers' planners): the source range starts
// on a 16-byte boundary and every stage copy is a multiple of 16 bytes; the
// source allocation extends at least 16 bytes past the last byte consumed
// (a short tail is rounded up to 16 bytes).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pj_device.cuh"

namespace pj {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase with the given parity.  Returns false (and
// raises ST_TIMEOUT) if it did not complete within SPIN_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* status)
{
    for (uint32_t i = 0; i < SPIN_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    raise_status(status, ST_TIMEOUT);
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Ring of NSTAGE stages of STAGE_BYTES each over the byte range
// [src, src + total_bytes).  Usage (all threads):
//   ring.start(...)   -- thread 0 issues the first copies
//   for (k = 0; k < ring.num_chunks(); ++k) {
//       const uint8_t* p = ring.wait(k);   // all threads
//       ... consume min(STAGE_BYTES, remaining) bytes at p ...
//       __syncthreads();
//       ring.release(k);                   // thread 0 refills the stage
//   }
//   ring.finish()                          // before the smem is reused
template <int NSTAGE, int STAGE_BYTES>
struct BulkRing {
    uint8_t* stages;   // NSTAGE * STAGE_BYTES, 16-byte aligned
    uint64_t* bars;    // NSTAGE mbarriers
    const uint8_t* src;
    int64_t total_bytes;
    uint32_t* status;
    uint32_t phase_bits;  // per-stage parity, identical in every thread
    int64_t issued;       // chunks issued (thread 0's view)

    __device__ __forceinline__ int64_t num_chunks() const
    {
        return (total_bytes + STAGE_BYTES - 1) / STAGE_BYTES;
    }

    // Must be followed by __syncthreads() before the first wait().
    __device__ __forceinline__ void init_barriers()
    {
        if (threadIdx.x == 0) {
            for (int s = 0; s < NSTAGE; ++s) mbar_init(&bars[s], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }

    __device__ __forceinline__ void issue(int64_t chunk)
    {
        const int s = static_cast<int>(chunk % NSTAGE);
        const int64_t off = chunk * STAGE_BYTES;
        int64_t len = total_bytes - off;
        if (len > STAGE_BYTES) len = STAGE_BYTES;
        const uint32_t bytes = static_cast<uint32_t>((len + 15) & ~int64_t(15));
        mbar_arrive_expect_tx(&bars[s], bytes);
        bulk_g2s(stages + static_cast<size_t>(s) * STAGE_BYTES, src + off, bytes, &bars[s]);
    }

    // Called by every thread with identical arguments; thread 0 issues.
    __device__ __forceinline__ void start(const void* src_, int64_t total_bytes_, uint32_t* status_)
    {
        src = static_cast<const uint8_t*>(src_);
        total_bytes = total_bytes_;
        status = status_;
        issued = 0;
        if (threadIdx.x == 0) {
            const int64_t n = num_chunks();
            for (; issued < n && issued < NSTAGE; ++issued) issue(issued);
        }
    }

    __device__ __forceinline__ const uint8_t* wait(int64_t chunk)
    {
        const int s = static_cast<int>(chunk % NSTAGE);
        mbar_wait(&bars[s], (phase_bits >> s) & 1u, status);
        phase_bits ^= 1u << s;
        return stages + static_cast<size_t>(s) * STAGE_BYTES;
    }

    // After a __syncthreads() that follows the last read of chunk `chunk`.
    __device__ __forceinline__ void release(int64_t chunk)
    {
        (void)chunk;
        if (threadIdx.x == 0 && issued < num_chunks()) {
            issue(issued);
            ++issued;
        }
    }
};

}  // namespace pj
