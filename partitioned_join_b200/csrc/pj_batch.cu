// pj_batch.cu -- many joins of uneven sizes in one batch.
//
// The reference runs one join per process (main.cu).  A batch of joins
// (pj_join_batch) is split by size:
//   * direct joins -- build side no larger than one shared-memory table --
//     skip partitioning altogether.  One persistent kernel drains a queue of
//     (join, probe chunk) work items: a CTA builds the join's table straight
//     from the raw build keys (bucket order; 4-byte entries holding a 16-bit
//     hash fingerprint and the build row, which fits 16 bits here), keeps it
//     while it takes further chunks of the same join, and probes.  A
//     fingerprint hit compares the raw build key (the build column is small
//     and stays in L2).  Matches go straight to the join's output at exact
//     positions (one atomic on the join's counter per warp step), so every
//     output is dense without a fix-up.
//   * larger joins (up to 2^10 partitions each) take the partitioned path
//     together (pj_internal::large_batch_*): one histogram, one scan and one
//     scatter launch over both key columns of all of them, then one work
//     split and one persistent join launch over all their partitions, each
//     match written at an exact position of its join's output.
//   * wider joins (or with large_batched = 0, every larger join) run the
//     partitioned path (pj_inner_join) one after the other in one reused
//     workspace region, their device status folded into the batch's.
// pj_batch_prepare writes the work table once (synchronous); pj_join_batch
// then only enqueues kernels, so it can be captured in a CUDA graph and
// replayed.  pj_batch_autotune measures candidate configurations on the
// batch itself.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pj.h"
#include "pj_device.cuh"
#include "pj_internal.h"

using namespace pj;

namespace {

struct BatchJob {
    const void* build;
    const void* probe;
    int64_t n_build;
    int64_t n_probe;
    int32_t* out_b;
    int32_t* out_p;
    int64_t capacity;
    unsigned long long* count;
    int64_t item_begin;  // first work item of this join
    int64_t items;       // its work items (probe chunks)
    int32_t nb_log2;     // log2 of its bucket count
    int32_t unique;
};

constexpr int DIRECT_MAX_BUILD = 40960;  // rows a direct table holds (16-bit row index, shared memory)
constexpr int DIRECT_NB_LOG2 = 14;       // most buckets of a direct table
constexpr int DIRECT_U = 4;              // probe rows per lane per step

// Buckets of a direct table for n_build rows: about two rows a bucket.
int nb_log2_for(int64_t n_build)
{
    int b = 1;
    while (b < DIRECT_NB_LOG2 && (int64_t(2) << b) <= std::max<int64_t>(2, n_build / 2)) ++b;
    return b;
}

// Direct-table shared memory: entries, then bucket ends (16-bit pairs).
size_t direct_smem(int max_build)
{
    return static_cast<size_t>(std::max(max_build, 1)) * 4 + (size_t(1) << nb_log2_for(max_build)) / 2 * 4;
}

// ---------------------------------------------------------------------------
// Device side.

__global__ void zero_counts_kernel(const BatchJob* __restrict__ jobs, int32_t n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) *jobs[i].count = 0;
}

__global__ void fold_status_kernel(const uint32_t* __restrict__ from, uint32_t* __restrict__ into)
{
    if (*from) atomicOr(into, *from);
}

template <typename K, int THREADS>
__global__ void __launch_bounds__(THREADS) batch_direct_kernel(const BatchJob* __restrict__ jobs, int32_t n_jobs,
                                                               int64_t total_items, int32_t chunk, int32_t max_build,
                                                               uint32_t* queue, uint32_t* status)
{
    constexpr int NW = THREADS / 32;
    constexpr int U = DIRECT_U;
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* tab = smem;              // fingerprint << 16 | build row
    uint32_t* ends = smem + max_build;  // bucket ends, 16-bit pairs
    __shared__ int64_t s_item;
    __shared__ int s_job;
    __shared__ uint32_t s_warp[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int cur = -1;

    for (;;) {
        __syncthreads();  // every warp is done with the previous item
        if (threadIdx.x == 0) {
            const int64_t it = static_cast<int64_t>(atomicAdd(queue, 1u));
            int j = -1;
            if (it < total_items) {  // last job with item_begin <= it
                int lo = 0, hi = n_jobs - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (jobs[mid].item_begin <= it) lo = mid; else hi = mid - 1;
                }
                j = lo;
            }
            s_item = it;
            s_job = j;
        }
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total_items) break;
        const int j = s_job;
        const BatchJob J = jobs[j];
        const K* __restrict__ bk = static_cast<const K*>(J.build);
        const K* __restrict__ pk = static_cast<const K*>(J.probe);
        const int nbl = J.nb_log2;
        const uint32_t nb_mask = (1u << nbl) - 1u;
        const int n_build = static_cast<int>(J.n_build);
        if (n_build > max_build) {  // prepare never queues such a join
            if (threadIdx.x == 0) raise_status(status, ST_OVERFLOW);
            continue;
        }
        if (j != cur) {
            // the join's table: count per bucket, scan, place
            const int nwords = (1 << nbl) / 2;
            for (int i = threadIdx.x; i < nwords; i += THREADS) ends[i] = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < n_build; i += THREADS) {
                const uint32_t b = hash_key(bk[i]) & nb_mask;
                atomicAdd(&ends[b >> 1], (b & 1u) ? 0x10000u : 1u);
            }
            __syncthreads();
            scan_u16_pairs<THREADS>(ends, nwords, s_warp);
            for (int i = threadIdx.x; i < n_build; i += THREADS) {
                const uint32_t h = hash_key(bk[i]);
                const uint32_t b = h & nb_mask;
                const uint32_t old = atomicAdd(&ends[b >> 1], (b & 1u) ? 0x10000u : 1u);
                const uint32_t pos = (b & 1u) ? (old >> 16) : (old & 0xffffu);
                tab[pos] = (((h >> nbl) & 0xffffu) << 16) | static_cast<uint32_t>(i);
            }
            __syncthreads();
            cur = j;
        }
        // probe the chunk: warps take steps of 32*U rows
        const int64_t lo = (item - J.item_begin) * chunk;
        const int64_t hi = lo + chunk < J.n_probe ? lo + chunk : J.n_probe;
        for (int64_t base = lo + static_cast<int64_t>(warp) * 32 * U; base < hi; base += NW * 32 * U) {
            K k[U];
            int32_t r[U];
            uint32_t fq[U];
            int at[U], end[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t i = base + u * 32 + lane;
                r[u] = i < hi ? static_cast<int32_t>(i) : -1;
                k[u] = r[u] >= 0 ? pk[i] : K(0);
                at[u] = end[u] = 0;
                fq[u] = 0;
                if (r[u] >= 0) {
                    const uint32_t h = hash_key(k[u]);
                    const uint32_t b = h & nb_mask;
                    fq[u] = (h >> nbl) & 0xffffu;
                    end[u] = static_cast<int>((ends[b >> 1] >> ((b & 1u) * 16)) & 0xffffu);
                    at[u] = b == 0 ? 0 : static_cast<int>((ends[(b - 1) >> 1] >> (((b - 1) & 1u) * 16)) & 0xffffu);
                }
            }
            // next verified match of tuple u from at[u], or -1
            auto next = [&](int u) -> int32_t {
                while (at[u] < end[u]) {
                    const uint32_t e = tab[at[u]++];
                    if ((e >> 16) == fq[u]) {
                        const int32_t row = static_cast<int32_t>(e & 0xffffu);
                        if (bk[row] == k[u]) return row;
                    }
                }
                return -1;
            };
            for (;;) {
                int32_t m[U];
                int c = 0;
                bool more = false;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    m[u] = next(u);
                    if (m[u] >= 0) {
                        ++c;
                        if (J.unique) at[u] = end[u];  // at most one match
                    }
                    more |= at[u] < end[u];
                }
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int n = __shfl_sync(0xffffffffu, incl, 31);
                if (n > 0) {
                    unsigned long long b0 = 0;
                    if (lane == 31) b0 = atomicAdd(J.count, static_cast<unsigned long long>(n));
                    b0 = __shfl_sync(0xffffffffu, b0, 31);
                    if (J.out_b) {
                        long long pos = static_cast<long long>(b0) + (incl - c);
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            if (m[u] >= 0) {
                                if (pos < J.capacity) {
                                    J.out_b[pos] = m[u];
                                    J.out_p[pos] = r[u];
                                } else {
                                    raise_status(status, ST_CAPACITY);
                                }
                                ++pos;
                            }
                        }
                    }
                }
                if (!__any_sync(0xffffffffu, more)) break;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Host side.

struct Split {
    std::vector<int> direct, large;
};

Split split_batch(const pj_join_desc* descs, int32_t n, const pj_batch_config& cfg)
{
    Split s;
    for (int i = 0; i < n; ++i) {
        const pj_join_desc& d = descs[i];
        if (d.n_build <= cfg.direct_max_build && d.n_build > 0 && d.n_probe > 0) s.direct.push_back(i);
        else s.large.push_back(i);
    }
    return s;
}

pj_plan large_plan(const pj_join_desc& d, const pj_batch_config& cfg, bool* ok)
{
    pj_plan p;
    *ok = pj_plan_default(&d, &p) == PJ_OK;
    if (*ok && cfg.large_bits_delta != 0) {
        pj_plan q = p;
        q.bits1 = std::max(0, p.bits1 + cfg.large_bits_delta);
        size_t b = 0;
        if (pj_workspace_size(&d, &q, &b) == PJ_OK) p = q;  // invalid tweaks keep the default
    }
    return p;
}

struct BatchLayout {
    size_t ctrl = 0, jobs = 0, large = 0, large_bytes = 0, batched = 0, total = 0;
    pj_internal::LargeBatch lb;  // the larger joins run together
    std::vector<int> sequential; // the larger joins run one after another
};

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

pj_status layout_for(const pj_join_desc* descs, int32_t n, const pj_batch_config& cfg, BatchLayout* L)
{
    BatchLayout b;
    b.ctrl = 0;
    b.jobs = 256;
    b.large = align256(b.jobs + sizeof(BatchJob) * static_cast<size_t>(std::max(n, 1)));
    const Split sp = split_batch(descs, n, cfg);
    if (cfg.large_batched) {
        pj_status s = pj_internal::large_batch_layout(descs, sp.large, cfg.large_bits_delta, &b.lb);
        if (s != PJ_OK) return s;
    }
    for (int i : sp.large)
        if (std::find(b.lb.joins.begin(), b.lb.joins.end(), i) == b.lb.joins.end()) b.sequential.push_back(i);
    for (int i : b.sequential) {
        const pj_join_desc& d = descs[i];
        bool ok = false;
        pj_plan p = large_plan(d, cfg, &ok);
        if (!ok) return PJ_ERR_INVALID;
        size_t w = 0;
        pj_status s = pj_workspace_size(&d, &p, &w);
        if (s != PJ_OK) return s;
        b.large_bytes = std::max(b.large_bytes, w);
    }
    b.batched = b.large + align256(b.large_bytes);
    b.total = b.batched + align256(b.lb.total);
    *L = std::move(b);
    return PJ_OK;
}

pj_status check_batch(const pj_join_desc* descs, const pj_output* outs, int32_t n, const pj_batch_config* cfg)
{
    if (!descs || n < 0 || !cfg) return PJ_ERR_INVALID;
    if (cfg->direct_threads != 256 && cfg->direct_threads != 512 && cfg->direct_threads != 1024) return PJ_ERR_INVALID;
    if (cfg->direct_chunk < 1024 || cfg->direct_max_build < 0 || cfg->direct_max_build > DIRECT_MAX_BUILD)
        return PJ_ERR_INVALID;
    if (cfg->large_bits_delta < -4 || cfg->large_bits_delta > 4) return PJ_ERR_INVALID;
    if (cfg->large_batched != 0 && cfg->large_batched != 1) return PJ_ERR_INVALID;
    for (int i = 0; i < n; ++i) {
        if (descs[i].key_bytes != descs[0].key_bytes) return PJ_ERR_INVALID;  // one key width per batch
        if (outs) {
            if (!outs[i].count || outs[i].capacity < 0) return PJ_ERR_INVALID;
            if (outs[i].capacity > 0 && (!outs[i].build_row || !outs[i].probe_row)) return PJ_ERR_INVALID;
        }
    }
    return PJ_OK;
}

int64_t direct_items(const pj_join_desc* descs, const Split& s, int chunk)
{
    int64_t t = 0;
    for (int i : s.direct) t += (descs[i].n_probe + chunk - 1) / chunk;
    return t;
}

template <typename K, int THREADS>
pj_status launch_direct(const BatchJob* jobs, int n_jobs, int64_t items, const pj_batch_config& cfg, uint32_t* queue,
                        uint32_t* status, cudaStream_t st)
{
    auto* kern = batch_direct_kernel<K, THREADS>;
    const size_t smem = direct_smem(cfg.direct_max_build);
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(kern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
        return PJ_ERR_CUDA;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, THREADS, smem);
    const int64_t grid = std::min<int64_t>(static_cast<int64_t>(sms) * std::max(per, 1), std::max<int64_t>(items, 1));
    kern<<<static_cast<unsigned>(grid), THREADS, smem, st>>>(jobs, n_jobs, items, cfg.direct_chunk, cfg.direct_max_build,
                                                            queue, status);
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

template <typename K>
pj_status launch_direct_k(const BatchJob* jobs, int n_jobs, int64_t items, const pj_batch_config& cfg, uint32_t* queue,
                          uint32_t* status, cudaStream_t st)
{
    switch (cfg.direct_threads) {
    case 256: return launch_direct<K, 256>(jobs, n_jobs, items, cfg, queue, status, st);
    case 512: return launch_direct<K, 512>(jobs, n_jobs, items, cfg, queue, status, st);
    default: return launch_direct<K, 1024>(jobs, n_jobs, items, cfg, queue, status, st);
    }
}

// parts: 1 = direct joins, 2 = large joins, 3 = both
pj_status run_batch(const pj_join_desc* descs, const pj_output* outs, int32_t n, const pj_batch_config& cfg, void* ws,
                    size_t ws_bytes, cudaStream_t st, int parts)
{
    BatchLayout L;
    pj_status s = layout_for(descs, n, cfg, &L);
    if (s != PJ_OK) return s;
    if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u) || ws_bytes < L.total) return PJ_ERR_WORKSPACE;
    uint8_t* w = static_cast<uint8_t*>(ws);
    uint32_t* status = reinterpret_cast<uint32_t*>(w + L.ctrl);
    uint32_t* queue = status + 1;
    if (cudaMemsetAsync(queue, 0, sizeof(uint32_t), st) != cudaSuccess) return PJ_ERR_CUDA;
    const Split sp = split_batch(descs, n, cfg);
    const BatchJob* jobs = reinterpret_cast<const BatchJob*>(w + L.jobs);
    if ((parts & 1) && !sp.direct.empty()) {
        const int nd = static_cast<int>(sp.direct.size());
        zero_counts_kernel<<<(nd + 255) / 256, 256, 0, st>>>(jobs, nd);
        const int64_t items = direct_items(descs, sp, cfg.direct_chunk);
        s = descs[0].key_bytes == 4 ? launch_direct_k<int32_t>(jobs, nd, items, cfg, queue, status, st)
                                    : launch_direct_k<int64_t>(jobs, nd, items, cfg, queue, status, st);
        if (s != PJ_OK) return s;
    }
    if (parts & 2) {
        if ((s = pj_internal::large_batch_run(L.lb, w + L.batched, status, st)) != PJ_OK) return s;
        void* lws = w + L.large;
        for (int i : L.sequential) {
            bool ok = false;
            const pj_plan p = large_plan(descs[i], cfg, &ok);
            pj_output o = outs[i];
            s = pj_inner_join(&descs[i], &p, &o, lws, L.large_bytes, st);
            if (s != PJ_OK) return s;
            fold_status_kernel<<<1, 1, 0, st>>>(static_cast<const uint32_t*>(lws), status);
        }
    }
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

}  // namespace

extern "C" {

pj_status pj_batch_config_default(int32_t key_bytes, pj_batch_config* cfg)
{
    if (!cfg || (key_bytes != 4 && key_bytes != 8)) return PJ_ERR_INVALID;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->direct_threads = 512;
    cfg->direct_chunk = 1 << 16;
    cfg->direct_max_build = key_bytes == 4 ? 20480 : 16384;
    cfg->large_bits_delta = 0;
    cfg->large_batched = 1;
    return PJ_OK;
}

pj_status pj_batch_workspace_size(const pj_join_desc* descs, int32_t n, const pj_batch_config* cfg, size_t* bytes)
{
    if (!bytes) return PJ_ERR_INVALID;
    pj_batch_config c;
    if (cfg) c = *cfg;
    else if (n > 0) pj_batch_config_default(descs[0].key_bytes, &c);
    else pj_batch_config_default(4, &c);
    pj_status s = check_batch(descs, nullptr, n, &c);
    if (s != PJ_OK) return s;
    BatchLayout L;
    if ((s = layout_for(descs, n, c, &L)) != PJ_OK) return s;
    *bytes = L.total;
    return PJ_OK;
}

pj_status pj_batch_prepare(const pj_join_desc* descs, const pj_output* outs, int32_t n, const pj_batch_config* cfg,
                           void* ws, size_t ws_bytes, pj_stream stream)
{
    pj_status s = check_batch(descs, outs, n, cfg);
    if (s != PJ_OK) return s;
    if (!outs && n > 0) return PJ_ERR_INVALID;
    BatchLayout L;
    if ((s = layout_for(descs, n, *cfg, &L)) != PJ_OK) return s;
    if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u) || ws_bytes < L.total) return PJ_ERR_WORKSPACE;
    const Split sp = split_batch(descs, n, *cfg);
    std::vector<BatchJob> jobs;
    int64_t item = 0;
    for (int i : sp.direct) {
        const pj_join_desc& d = descs[i];
        BatchJob j{};
        j.build = d.build_keys;
        j.probe = d.probe_keys;
        j.n_build = d.n_build;
        j.n_probe = d.n_probe;
        j.out_b = outs[i].build_row;
        j.out_p = outs[i].probe_row;
        j.capacity = outs[i].capacity;
        j.count = reinterpret_cast<unsigned long long*>(outs[i].count);
        j.items = (d.n_probe + cfg->direct_chunk - 1) / cfg->direct_chunk;
        j.item_begin = item;
        j.nb_log2 = nb_log2_for(d.n_build);
        j.unique = d.unique_build_keys ? 1 : 0;
        item += j.items;
        jobs.push_back(j);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    if (cudaMemsetAsync(w + L.ctrl, 0, 256, st) != cudaSuccess) return PJ_ERR_CUDA;
    if (!jobs.empty() &&
        cudaMemcpyAsync(w + L.jobs, jobs.data(), sizeof(BatchJob) * jobs.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return PJ_ERR_CUDA;
    if ((s = pj_internal::large_batch_upload(L.lb, outs, w + L.batched, st)) != PJ_OK) return s;
    return cudaStreamSynchronize(st) == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

pj_status pj_join_batch(const pj_join_desc* descs, const pj_output* outs, int32_t n, const pj_batch_config* cfg,
                        void* ws, size_t ws_bytes, pj_stream stream)
{
    pj_status s = check_batch(descs, outs, n, cfg);
    if (s != PJ_OK) return s;
    if (!outs && n > 0) return PJ_ERR_INVALID;
    return run_batch(descs, outs, n, *cfg, ws, ws_bytes, static_cast<cudaStream_t>(stream), 3);
}

pj_status pj_batch_check(void* ws, pj_stream stream)
{
    if (!ws) return PJ_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaStreamSynchronize(st) != cudaSuccess) return PJ_ERR_CUDA;
    uint32_t v = 0;
    if (cudaMemcpy(&v, ws, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return PJ_ERR_CUDA;
    const uint32_t zero = 0;
    if (cudaMemcpy(ws, &zero, sizeof(zero), cudaMemcpyHostToDevice) != cudaSuccess) return PJ_ERR_CUDA;
    if (v & ST_INTERNAL) return PJ_ERR_INTERNAL;
    if (v & ST_TIMEOUT) return PJ_ERR_TIMEOUT;
    if (v & ST_OVERFLOW) return PJ_ERR_OVERFLOW;
    if (v & ST_CAPACITY) return PJ_ERR_CAPACITY;
    return PJ_OK;
}

pj_status pj_batch_autotune(const pj_join_desc* descs, const pj_output* outs, int32_t n, void* ws, size_t ws_bytes,
                            pj_stream stream, pj_batch_config* best, float* best_ms)
{
    if (!best || n <= 0 || !descs || !outs) return PJ_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return PJ_ERR_CUDA;
    // time one configuration: prepare, one warm run, then the better of two
    auto time_cfg = [&](const pj_batch_config& c, int parts, float* ms) -> pj_status {
        size_t need = 0;
        pj_status s = pj_batch_workspace_size(descs, n, &c, &need);
        if (s != PJ_OK) return s;
        if (need > ws_bytes) return PJ_ERR_WORKSPACE;
        if ((s = pj_batch_prepare(descs, outs, n, &c, ws, ws_bytes, stream)) != PJ_OK) return s;
        float bestv = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, st);
            if ((s = run_batch(descs, outs, n, c, ws, ws_bytes, st, parts)) != PJ_OK) return s;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) return PJ_ERR_CUDA;
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) bestv = std::min(bestv, t);
        }
        if ((s = pj_batch_check(ws, stream)) != PJ_OK) return s;
        *ms = bestv;
        return PJ_OK;
    };
    pj_batch_config base;
    pj_batch_config_default(descs[0].key_bytes, &base);
    pj_batch_config cur = base;
    float cur_ms = 0;
    pj_status s = time_cfg(cur, 3, &cur_ms);
    // 1. where the direct path ends (whole batch timed)
    const int limits[] = {0, 4096, 8192, 16384, 24576, DIRECT_MAX_BUILD};
    for (int lim : limits) {
        if (s != PJ_OK) break;
        pj_batch_config c = cur;
        c.direct_max_build = lim;
        float t = 0;
        const pj_status r = time_cfg(c, 3, &t);
        if (r == PJ_OK && t < cur_ms) {
            cur = c;
            cur_ms = t;
        }
    }
    // 2. block size and chunk of the direct kernel (direct part timed)
    if (s == PJ_OK && cur.direct_max_build > 0) {
        float dbest = 0;
        if (time_cfg(cur, 1, &dbest) == PJ_OK) {
            for (int th : {256, 512, 1024})
                for (int ch : {1 << 14, 1 << 16, 1 << 18}) {
                    pj_batch_config c = cur;
                    c.direct_threads = th;
                    c.direct_chunk = ch;
                    float t = 0;
                    if (time_cfg(c, 1, &t) == PJ_OK && t < dbest) {
                        dbest = t;
                        cur.direct_threads = th;
                        cur.direct_chunk = ch;
                    }
                }
        }
    }
    // 3. radix width of the partitioned joins, and whether they run
    //    together or one after another (large part timed)
    if (s == PJ_OK) {
        float lbest = 0;
        if (time_cfg(cur, 2, &lbest) == PJ_OK) {
            for (int together : {1, 0})
                for (int dlt : {-1, 0, 1}) {
                    if (together == cur.large_batched && dlt == cur.large_bits_delta) continue;
                    pj_batch_config c = cur;
                    c.large_bits_delta = dlt;
                    c.large_batched = together;
                    float t = 0;
                    if (time_cfg(c, 2, &t) == PJ_OK && t < lbest) {
                        lbest = t;
                        cur.large_bits_delta = dlt;
                        cur.large_batched = together;
                    }
                }
        }
    }
    if (s == PJ_OK) {
        s = time_cfg(cur, 3, &cur_ms);
        *best = cur;
        if (best_ms) *best_ms = cur_ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

}  // extern "C"
