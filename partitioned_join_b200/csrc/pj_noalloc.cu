// pj_noalloc.cu -- pj_inner_join_noalloc: the join for callers that cannot
// allocate device memory.  Its workspace is one fixed array in the library's
// own device memory instead of a buffer the caller passes in.
//
// Who needs it: a host runtime that binds the join through a thin FFI and owns
// no device allocator (it only holds the key and output columns it was
// handed), and callers that must not call cudaMalloc/cudaFree around a join
// because cudaFree waits for the whole device and would stall unrelated
// streams.  Such callers are limited to joins whose workspace fits
// PJ_NOALLOC_SCRATCH_BYTES (64 MiB: about 2^20 build x 2^22 probe 4-byte keys
// under the default plan).  Larger joins are rejected with PJ_ERR_WORKSPACE
// before any device work; they need pj_inner_join and a workspace of
// pj_workspace_size() bytes.
//
// Nothing in the scratch has to start at zero: pj_inner_join clears the
// counters and status word it uses at the start of every call, and the
// status is read back and cleared before this call returns.
//
// The scratch is one array per device, shared by every caller in the
// process.  Two calls on the same device that overlap in time (from two host
// threads, whatever their streams) write the same scratch and race; callers
// must serialise them.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/pj.h"

namespace {

static_assert(PJ_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size must keep 256-byte granularity");

// The workspace of pj_inner_join_noalloc on each device.  The module that holds
// it loads on the first call on a device, so processes that never call
// pj_inner_join_noalloc do not reserve it (with the default lazy module loading).
static __device__ __align__(256) unsigned char g_noalloc_scratch[PJ_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;

// Device address of g_noalloc_scratch on the current device, looked up once per
// device.  The first lookup loads this file's module on that device, which is
// why the first call on each device must not happen during stream capture.
pj_status scratch_address(void** ptr)
{
    static std::mutex mu;
    static void* cache[MAX_DEVICES] = {};
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return PJ_ERR_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) return PJ_ERR_INVALID;
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return PJ_ERR_CUDA;
        }
        if (reinterpret_cast<uintptr_t>(p) % 256 != 0) return PJ_ERR_WORKSPACE;
        cache[dev] = p;
    }
    *ptr = cache[dev];
    return PJ_OK;
}

}  // namespace

extern "C" pj_status pj_inner_join_noalloc(const pj_join_desc* desc, const pj_plan* plan, pj_output* out,
                                           pj_stream stream)
{
    size_t need = 0;
    pj_status s = pj_workspace_size(desc, plan, &need);
    if (s != PJ_OK) return s;
    if (need > PJ_NOALLOC_SCRATCH_BYTES) return PJ_ERR_WORKSPACE;
    void* ws = nullptr;
    if ((s = scratch_address(&ws)) != PJ_OK) return s;
    s = pj_inner_join(desc, plan, out, ws, PJ_NOALLOC_SCRATCH_BYTES, stream);
    // Arguments rejected before any launch leave nothing on the device to
    // wait for.  After a launch (or a launch that failed part-way), pj_check
    // waits for the join and clears the status word, so the next call starts
    // clean.
    if (s != PJ_OK && s != PJ_ERR_CUDA) return s;
    const pj_status device_status = pj_check(ws, stream);
    return s != PJ_OK ? s : device_status;
}
