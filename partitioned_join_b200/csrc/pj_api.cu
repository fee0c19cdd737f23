// pj_api.cu -- host side of the C ABI in include/pj.h: planning, workspace
// layout and the stage sequence (the reference's main.cu:762-892).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/pj.h"
#include "pj_device.cuh"
#include "pj_join.cuh"
#include "pj_partition.cuh"

using namespace pj;

namespace {

// ---------------------------------------------------------------------------
// Fixed kernel configurations.
constexpr int SC_THREADS = 1024;
constexpr int SC_NSTAGE = 3;
constexpr int SC_V32 = 4, SC_V64 = 2;   // keys per thread per round: 16 KB stages
constexpr int SC_W32 = 4, SC_W64 = 8;   // tuples per write-combining buffer: 32 B / 96 B
constexpr int JN_THREADS = 1024;
constexpr int JN_OB = 4096;
constexpr int JN_NSTAGE = 3;
constexpr int JN_STAGE_TUPLES = 2048;
constexpr int MAX_SPLIT_LOG2 = 6;

struct DevInfo {
    int device = -1;
    int sms = 0;
    size_t smem_optin = 0;
};

DevInfo dev_info()
{
    static std::mutex mu;
    static DevInfo cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DevInfo{};
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && cache[dev].device == dev) return cache[dev];
    DevInfo d;
    d.device = dev;
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    d.sms = v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    d.smem_optin = static_cast<size_t>(v);
    if (dev >= 0 && dev < 64) cache[dev] = d;
    return d;
}

// The planner must work without a GPU (sizes only): assume a B200 when no
// device is visible.
int sm_count()
{
    const DevInfo d = dev_info();
    return d.sms > 0 ? d.sms : 148;
}

size_t smem_limit()
{
    const DevInfo d = dev_info();
    return d.smem_optin > 0 ? d.smem_optin : 232448;
}

int ilog2_ceil(int64_t x)
{
    int b = 0;
    while ((int64_t(1) << b) < x) ++b;
    return b;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename K>
constexpr int sc_v() { return sizeof(K) == 4 ? SC_V32 : SC_V64; }
template <typename K>
constexpr int sc_w() { return sizeof(K) == 4 ? SC_W32 : SC_W64; }

template <typename K>
size_t scatter_smem(int P)
{
    return ScatterSmem<K, SC_THREADS, sc_v<K>(), sc_w<K>(), SC_NSTAGE>::bytes(P);
}

template <typename K>
size_t join_smem(int T)
{
    return JoinSmem<K, JN_THREADS, JN_OB, JN_NSTAGE, JN_STAGE_TUPLES>::bytes(T);
}

int max_one_pass_bits(int key_bytes)
{
    int b = 0;
    const size_t lim = smem_limit();
    for (int t = 1; t <= 16; ++t) {
        const size_t s = key_bytes == 4 ? scatter_smem<int32_t>(1 << t) : scatter_smem<int64_t>(1 << t);
        if (s <= lim) b = t;
    }
    return b;
}

int max_table_slots(int key_bytes)
{
    const size_t lim = smem_limit();
    const size_t base = key_bytes == 4 ? join_smem<int32_t>(0) : join_smem<int64_t>(0);
    const int slot = key_bytes == 4 ? 8 : 12;
    if (lim <= base + 1024) return 0;
    int T = static_cast<int>((lim - base - 512) / slot);
    return T & ~127;
}

bool valid_desc(const pj_join_desc* d)
{
    if (!d) return false;
    if (d->key_bytes != 4 && d->key_bytes != 8) return false;
    if (d->n_build < 0 || d->n_probe < 0 || d->n_build > INT32_MAX || d->n_probe > INT32_MAX) return false;
    if (d->n_build > 0 && !d->build_keys) return false;
    if (d->n_probe > 0 && !d->probe_keys) return false;
    if (d->payload_bytes != 0 && d->payload_bytes != 4 && d->payload_bytes != 8) return false;
    return true;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

pj_status check_plan(const pj_join_desc* d, const pj_plan* p)
{
    if (p->passes != 1) return PJ_ERR_INVALID;
    if (p->bits1 < 0 || p->bits1 > max_one_pass_bits(d->key_bytes)) return PJ_ERR_INVALID;
    if (p->digit_mode != PJ_DIGIT_RAW && p->digit_mode != PJ_DIGIT_HASH) return PJ_ERR_INVALID;
    if (p->slot_mode != PJ_SLOT_FAST && p->slot_mode != PJ_SLOT_REF) return PJ_ERR_INVALID;
    if (p->split_mode != PJ_SPLIT_HASH && p->split_mode != PJ_SPLIT_POSITION) return PJ_ERR_INVALID;
    if (p->table_slots < 64 || p->table_slots > max_table_slots(d->key_bytes)) return PJ_ERR_INVALID;
    if (p->probe_chunk < 16 || (p->probe_chunk & 15)) return PJ_ERR_INVALID;
    if (!(p->max_fill > 0.05f && p->max_fill <= 0.95f)) return PJ_ERR_INVALID;
    const int used = (p->digit_mode == PJ_DIGIT_HASH ? p->bits1 + p->bits2 : 0) + MAX_SPLIT_LOG2;
    if (used > 26) return PJ_ERR_INVALID;
    return PJ_OK;
}

// ---------------------------------------------------------------------------
// Workspace layout.  Everything 256-byte aligned.
struct Layout {
    int P = 1;
    int b_items = 1, p_items = 1;
    int64_t b_chunk = 16, p_chunk = 16;
    int64_t b_cap = 0, p_cap = 0;  // tuples
    size_t status = 0, counters = 0, b_tiles = 0, p_tiles = 0, i_tiles = 0, b_tot = 0, p_tot = 0, ctrl_end = 0;
    size_t b_counts = 0, p_counts = 0, b_off = 0, p_off = 0, split = 0, items = 0, item_off = 0;
    size_t b_tuples = 0, p_tuples = 0, total = 0;
    int64_t b_tiles_n = 0, p_tiles_n = 0, i_tiles_n = 0;
};

constexpr int CTR_QUEUE = 0, CTR_BTILE = 1, CTR_PTILE = 2, CTR_ITILE = 3;

int64_t chunk_for(int64_t n, int items)
{
    int64_t c = (n + items - 1) / std::max(items, 1);
    c = (c + 15) / 16 * 16;
    return std::max<int64_t>(c, 16);
}

int scatter_items(const pj_plan* p) { return sm_count() * std::max(1, p->scatter_ctas_per_sm); }

int64_t part_capacity(int64_t n, int key_bytes, int P, int items)
{
    const int W = key_bytes == 4 ? SC_W32 : SC_W64;
    return n + static_cast<int64_t>(items) * P * (W - 1) + W;
}

Layout make_layout(const pj_join_desc* d, const pj_plan* p)
{
    Layout L;
    L.P = 1 << p->bits1;
    L.b_items = L.p_items = scatter_items(p);
    L.b_chunk = chunk_for(d->n_build, L.b_items);
    L.p_chunk = chunk_for(d->n_probe, L.p_items);
    L.b_cap = part_capacity(d->n_build, d->key_bytes, L.P, L.b_items);
    L.p_cap = part_capacity(d->n_probe, d->key_bytes, L.P, L.p_items);
    const int64_t mb = static_cast<int64_t>(L.P) * L.b_items, mp = static_cast<int64_t>(L.P) * L.p_items;
    L.b_tiles_n = (mb + SCAN_TILE - 1) / SCAN_TILE + 1;
    L.p_tiles_n = (mp + SCAN_TILE - 1) / SCAN_TILE + 1;
    L.i_tiles_n = (L.P + SCAN_TILE - 1) / SCAN_TILE + 1;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = align_up(o + bytes, 256); return at; };
    // control block: zeroed at the start of every call
    L.status = take(4);
    L.counters = take(4 * 8);
    L.b_tiles = take(8 * L.b_tiles_n);
    L.p_tiles = take(8 * L.p_tiles_n);
    L.i_tiles = take(8 * L.i_tiles_n);
    L.b_tot = take(4 * static_cast<size_t>(L.P));
    L.p_tot = take(4 * static_cast<size_t>(L.P));
    L.ctrl_end = o;
    L.b_counts = take(4 * static_cast<size_t>(mb));
    L.p_counts = take(4 * static_cast<size_t>(mp));
    L.b_off = take(8 * static_cast<size_t>(mb + 1));
    L.p_off = take(8 * static_cast<size_t>(mp + 1));
    L.split = take(4 * static_cast<size_t>(L.P));
    L.items = take(8 * static_cast<size_t>(L.P));
    L.item_off = take(8 * static_cast<size_t>(L.P + 1));
    const int TW = d->key_bytes == 4 ? 2 : 3;
    L.b_tuples = take(4 * static_cast<size_t>(TW) * L.b_cap + 64);
    L.p_tuples = take(4 * static_cast<size_t>(TW) * L.p_cap + 64);
    L.total = o;
    return L;
}

DigitFn digit_fn(int mode, int bits_before, int bits, int raw_shift)
{
    DigitFn f;
    f.mode = mode;
    f.mask = bits > 0 ? (1u << bits) - 1u : 0u;
    f.shift = mode == PJ_DIGIT_HASH ? (bits > 0 ? 32 - bits_before - bits : 0) : raw_shift;
    return f;
}

#define PJ_CUDA(call)                                            \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) {                                 \
            last_cuda_error() = e_;                              \
            return PJ_ERR_CUDA;                                  \
        }                                                        \
    } while (0)

cudaError_t& last_cuda_error()
{
    static thread_local cudaError_t e = cudaSuccess;
    return e;
}

template <typename F>
cudaError_t set_smem(F* fn, size_t bytes)
{
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(bytes));
}

// ---------------------------------------------------------------------------
// Small elementwise kernels of the stage entry points.
template <typename K>
__global__ void hash_keys_kernel(const K* __restrict__ keys, int64_t n, uint32_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = hash_key(keys[i]);
}

template <typename K>
__global__ void hash_slots_kernel(const K* __restrict__ keys, int64_t n, int32_t T, int32_t ref, int32_t skip,
                                  int32_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const uint32_t h = hash_key(keys[i]);
        out[i] = static_cast<int32_t>(ref ? slot_ref(h, T) : slot_fast(h, skip, static_cast<uint32_t>(T)));
    }
}

// Partition boundaries from the flattened segment offsets: part[p] = off[p*items].
__global__ void partition_bounds_kernel(const int64_t* __restrict__ off, int32_t items, int32_t P,
                                        int64_t* __restrict__ part)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p <= P) part[p] = off[static_cast<int64_t>(p) * items];
}

unsigned grid_for(int64_t n, int threads)
{
    const int64_t g = (n + threads - 1) / threads;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(g, static_cast<int64_t>(sm_count()) * 32)));
}

// ---------------------------------------------------------------------------
// Stage launchers.

template <typename K>
pj_status launch_hist(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P, uint32_t* counts,
                      int32_t* totals, uint32_t* status, cudaStream_t st)
{
    const size_t smem = static_cast<size_t>(HIST_NSTAGE) * HIST_THREADS * HIST_V * sizeof(K) + 4 * static_cast<size_t>(P);
    PJ_CUDA(set_smem(hist_keys_kernel<K>, smem));
    hist_keys_kernel<K><<<items, HIST_THREADS, smem, st>>>(keys, n, chunk, items, f, P, counts, totals, status);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename TIn>
pj_status launch_scan(const TIn* in, int64_t m, uint32_t round_to, int64_t* out, uint64_t* tiles,
                      uint32_t* tile_counter, uint32_t* status, cudaStream_t st)
{
    const int64_t ntiles = std::max<int64_t>(1, (m + SCAN_TILE - 1) / SCAN_TILE);
    lookback_scan_kernel<TIn><<<static_cast<unsigned>(ntiles), SCAN_THREADS, 0, st>>>(in, m, round_to, out, tiles,
                                                                                    tile_counter, status);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K>
pj_status launch_scatter(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P,
                         const int64_t* offsets, uint32_t* out, int64_t out_cap, uint32_t* status, cudaStream_t st)
{
    constexpr int V = sc_v<K>(), W = sc_w<K>();
    auto* kern = scatter_keys_kernel<K, SC_THREADS, V, W, SC_NSTAGE>;
    const size_t smem = scatter_smem<K>(P);
    PJ_CUDA(set_smem(kern, smem));
    kern<<<items, SC_THREADS, smem, st>>>(keys, n, chunk, items, f, P, offsets, out,
                                         static_cast<uint32_t>(std::min<int64_t>(out_cap, UINT32_MAX)), status);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K, bool UNIQUE, bool HASH_SPLIT, bool SLOT_REF>
pj_status launch_join_t(const JoinArgs& a, cudaStream_t st)
{
    auto* kern = join_kernel<K, UNIQUE, HASH_SPLIT, SLOT_REF, JN_THREADS, JN_OB, JN_NSTAGE, JN_STAGE_TUPLES>;
    const size_t smem = join_smem<K>(a.table_slots);
    PJ_CUDA(set_smem(kern, smem));
    int per_sm = 0;
    PJ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, JN_THREADS, smem));
    per_sm = std::max(per_sm, 1);
    kern<<<sm_count() * per_sm, JN_THREADS, smem, st>>>(a);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K>
pj_status launch_join(const JoinArgs& a, bool unique, bool hash_split, bool slot_ref, cudaStream_t st)
{
    if (unique) {
        if (hash_split)
            return slot_ref ? launch_join_t<K, true, true, true>(a, st) : launch_join_t<K, true, true, false>(a, st);
        return slot_ref ? launch_join_t<K, true, false, true>(a, st) : launch_join_t<K, true, false, false>(a, st);
    }
    if (hash_split)
        return slot_ref ? launch_join_t<K, false, true, true>(a, st) : launch_join_t<K, false, true, false>(a, st);
    return slot_ref ? launch_join_t<K, false, false, true>(a, st) : launch_join_t<K, false, false, false>(a, st);
}

// Partition one side: histogram -> scan -> scatter.
template <typename K>
pj_status partition_side(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P, uint32_t* counts,
                         int32_t* totals, int64_t* off, uint64_t* tiles, uint32_t* tile_ctr, uint32_t* out,
                         int64_t out_cap, uint32_t* status, cudaStream_t st)
{
    pj_status s;
    if ((s = launch_hist<K>(keys, n, chunk, items, f, P, counts, totals, status, st)) != PJ_OK) return s;
    if ((s = launch_scan<uint32_t>(counts, static_cast<int64_t>(P) * items, static_cast<uint32_t>(sc_w<K>()), off,
                                   tiles, tile_ctr, status, st)) != PJ_OK)
        return s;
    return launch_scatter<K>(keys, n, chunk, items, f, P, off, out, out_cap, status, st);
}

// Optional stage events: ev[i] is recorded before stage i, ev[PJ_STAGE_TOTAL] at the end.
struct StageEvents {
    cudaEvent_t* ev = nullptr;
    void mark(int i, cudaStream_t st) const
    {
        if (ev) cudaEventRecord(ev[i], st);
    }
};

template <typename K>
pj_status run_join(const pj_join_desc* d, const pj_plan* p, const Layout& L, uint8_t* ws, int32_t* out_b,
                   int32_t* out_p, int64_t capacity, int64_t* count, cudaStream_t st,
                   const StageEvents& E = StageEvents())
{
    uint32_t* status = reinterpret_cast<uint32_t*>(ws + L.status);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(ws + L.counters);
    PJ_CUDA(cudaMemsetAsync(ws, 0, L.ctrl_end, st));
    PJ_CUDA(cudaMemsetAsync(count, 0, sizeof(int64_t), st));
    if (d->n_build == 0 || d->n_probe == 0) {
        for (int i = 0; i < PJ_NUM_STAGES; ++i) E.mark(i, st);
        return PJ_OK;
    }

    const DigitFn f = digit_fn(p->digit_mode, 0, p->bits1, 0);
    pj_status s;
    for (int side = 0; side < 2; ++side) {
        const K* keys = static_cast<const K*>(side == 0 ? d->build_keys : d->probe_keys);
        const int64_t n = side == 0 ? d->n_build : d->n_probe;
        const int64_t chunk = side == 0 ? L.b_chunk : L.p_chunk;
        const int items = side == 0 ? L.b_items : L.p_items;
        uint32_t* counts = reinterpret_cast<uint32_t*>(ws + (side == 0 ? L.b_counts : L.p_counts));
        int32_t* tot = reinterpret_cast<int32_t*>(ws + (side == 0 ? L.b_tot : L.p_tot));
        int64_t* off = reinterpret_cast<int64_t*>(ws + (side == 0 ? L.b_off : L.p_off));
        uint64_t* tiles = reinterpret_cast<uint64_t*>(ws + (side == 0 ? L.b_tiles : L.p_tiles));
        uint32_t* tuples = reinterpret_cast<uint32_t*>(ws + (side == 0 ? L.b_tuples : L.p_tuples));
        const int64_t cap = side == 0 ? L.b_cap : L.p_cap;
        const int st0 = side == 0 ? PJ_STAGE_BUILD_HIST : PJ_STAGE_PROBE_HIST;
        E.mark(st0, st);
        if ((s = launch_hist<K>(keys, n, chunk, items, f, L.P, counts, tot, status, st)) != PJ_OK) return s;
        E.mark(st0 + 1, st);
        if ((s = launch_scan<uint32_t>(counts, static_cast<int64_t>(L.P) * items, static_cast<uint32_t>(sc_w<K>()),
                                       off, tiles, ctr + (side == 0 ? CTR_BTILE : CTR_PTILE), status, st)) != PJ_OK)
            return s;
        E.mark(st0 + 2, st);
        if ((s = launch_scatter<K>(keys, n, chunk, items, f, L.P, off, tuples, cap, status, st)) != PJ_OK) return s;
    }
    E.mark(PJ_STAGE_JOIN_PLAN, st);

    const int cap_per_table = std::max(1, static_cast<int>(p->table_slots * p->max_fill));
    const bool hash_split = p->split_mode == PJ_SPLIT_HASH;
    join_items_kernel<<<(L.P + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<int64_t*>(ws + L.b_off), reinterpret_cast<int64_t*>(ws + L.p_off), L.b_items, L.p_items,
        L.P, reinterpret_cast<int32_t*>(ws + L.b_tot), reinterpret_cast<int32_t*>(ws + L.p_tot), cap_per_table,
        p->probe_chunk, hash_split ? 1 : 0, MAX_SPLIT_LOG2, reinterpret_cast<int32_t*>(ws + L.split),
        reinterpret_cast<int64_t*>(ws + L.items), status);
    PJ_CUDA(cudaGetLastError());
    if ((s = launch_scan<int64_t>(reinterpret_cast<int64_t*>(ws + L.items), L.P, 1u,
                                  reinterpret_cast<int64_t*>(ws + L.item_off), reinterpret_cast<uint64_t*>(ws + L.i_tiles),
                                  ctr + CTR_ITILE, status, st)) != PJ_OK)
        return s;

    JoinArgs a{};
    a.build_tuples = reinterpret_cast<const uint32_t*>(ws + L.b_tuples);
    a.probe_tuples = reinterpret_cast<const uint32_t*>(ws + L.p_tuples);
    a.build_off = reinterpret_cast<const int64_t*>(ws + L.b_off);
    a.probe_off = reinterpret_cast<const int64_t*>(ws + L.p_off);
    a.b_items = L.b_items;
    a.p_items = L.p_items;
    a.P = L.P;
    a.digit_bits = p->digit_mode == PJ_DIGIT_HASH ? p->bits1 + p->bits2 : 0;
    a.split_log2 = reinterpret_cast<const int32_t*>(ws + L.split);
    a.item_off = reinterpret_cast<const int64_t*>(ws + L.item_off);
    a.queue = ctr + CTR_QUEUE;
    a.table_slots = p->table_slots;
    a.probe_chunk = p->probe_chunk;
    a.position_chunk = std::max(16, cap_per_table / 16 * 16);
    a.out_build = out_b;
    a.out_probe = out_p;
    a.capacity = capacity;
    a.count = reinterpret_cast<unsigned long long*>(count);
    a.status = status;
    E.mark(PJ_STAGE_JOIN, st);
    s = launch_join<K>(a, d->unique_build_keys != 0, hash_split, p->slot_mode == PJ_SLOT_REF, st);
    E.mark(PJ_STAGE_TOTAL, st);
    return s;
}

pj_status resolve_plan(const pj_join_desc* d, const pj_plan* in, pj_plan* out)
{
    if (in) *out = *in;
    else {
        pj_status s = pj_plan_default(d, out);
        if (s != PJ_OK) return s;
    }
    return check_plan(d, out);
}

}  // namespace

// ===========================================================================
extern "C" {

const char* pj_status_string(pj_status s)
{
    switch (s) {
    case PJ_OK: return "ok";
    case PJ_ERR_INVALID: return "invalid argument";
    case PJ_ERR_CAPACITY: return "output capacity too small";
    case PJ_ERR_CUDA: return "CUDA runtime error";
    case PJ_ERR_TIMEOUT: return "device-side wait timed out";
    case PJ_ERR_WORKSPACE: return "workspace missing, misaligned or too small";
    case PJ_ERR_OVERFLOW: return "shared-memory table overflow (plan too coarse)";
    case PJ_ERR_ALIGNMENT: return "input column not 16-byte aligned";
    case PJ_ERR_INTERNAL: return "device-side consistency check failed";
    }
    return "unknown status";
}

const char* pj_version(void) { return "partitioned_join_b200 0.1 (sm_100a)"; }

pj_status pj_plan_default(const pj_join_desc* d, pj_plan* p)
{
    if (!valid_desc(d) || !p) return PJ_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->passes = 1;
    p->digit_mode = PJ_DIGIT_HASH;
    p->slot_mode = PJ_SLOT_FAST;
    p->split_mode = d->unique_build_keys ? PJ_SPLIT_HASH : PJ_SPLIT_POSITION;
    p->max_fill = 0.5f;  // HASH_TABLE_OCC, hash_join_kernels.cuh:21
    p->table_slots = d->key_bytes == 4 ? 16384 : 8192;
    p->table_slots = std::min(p->table_slots, max_table_slots(d->key_bytes));
    p->join_threads = JN_THREADS;
    p->scatter_threads = SC_THREADS;
    p->scatter_ctas_per_sm = 1;
    p->probe_chunk = 1 << 16;
    const int64_t cap = static_cast<int64_t>(p->table_slots * p->max_fill);
    const int want = ilog2_ceil(std::max<int64_t>(1, (d->n_build + cap - 1) / cap));
    p->bits1 = std::min(want, max_one_pass_bits(d->key_bytes));
    p->bits2 = 0;
    return PJ_OK;
}

pj_status pj_workspace_size(const pj_join_desc* d, const pj_plan* plan, size_t* bytes)
{
    if (!valid_desc(d) || !bytes) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = resolve_plan(d, plan, &p);
    if (s != PJ_OK) return s;
    *bytes = make_layout(d, &p).total;
    return PJ_OK;
}

static pj_status check_ws(const pj_join_desc* d, const pj_plan* p, void* ws, size_t ws_bytes, Layout* L)
{
    *L = make_layout(d, p);
    if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u) || ws_bytes < L->total) return PJ_ERR_WORKSPACE;
    return PJ_OK;
}

static pj_status check_inputs(const pj_join_desc* d)
{
    if (d->n_build > 0 && !aligned16(d->build_keys)) return PJ_ERR_ALIGNMENT;
    if (d->n_probe > 0 && !aligned16(d->probe_keys)) return PJ_ERR_ALIGNMENT;
    return PJ_OK;
}

pj_status pj_inner_join(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws, size_t ws_bytes,
                        pj_stream stream)
{
    if (!valid_desc(d) || !out || !out->count || out->capacity < 0) return PJ_ERR_INVALID;
    if (out->capacity > 0 && (!out->build_row || !out->probe_row)) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = resolve_plan(d, plan, &p);
    if (s != PJ_OK) return s;
    if ((s = check_inputs(d)) != PJ_OK) return s;
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    if (d->key_bytes == 4) return run_join<int32_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st);
    return run_join<int64_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st);
}

pj_status pj_inner_join_timed(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws,
                              size_t ws_bytes, pj_stream stream, float* stage_ms)
{
    if (!valid_desc(d) || !out || !out->count || out->capacity < 0 || !stage_ms) return PJ_ERR_INVALID;
    if (out->capacity > 0 && (!out->build_row || !out->probe_row)) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = resolve_plan(d, plan, &p);
    if (s != PJ_OK) return s;
    if ((s = check_inputs(d)) != PJ_OK) return s;
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[PJ_NUM_STAGES];
    for (int i = 0; i < PJ_NUM_STAGES; ++i) PJ_CUDA(cudaEventCreate(&ev[i]));
    StageEvents E;
    E.ev = ev;
    uint8_t* w = static_cast<uint8_t*>(ws);
    if (d->key_bytes == 4)
        s = run_join<int32_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st, E);
    else
        s = run_join<int64_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st, E);
    cudaError_t e = cudaStreamSynchronize(st);
    if (s == PJ_OK && e == cudaSuccess) {
        for (int i = 0; i + 1 < PJ_NUM_STAGES; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
        cudaEventElapsedTime(&stage_ms[PJ_STAGE_TOTAL], ev[0], ev[PJ_STAGE_TOTAL]);
    }
    for (int i = 0; i < PJ_NUM_STAGES; ++i) cudaEventDestroy(ev[i]);
    if (s == PJ_OK && e != cudaSuccess) {
        last_cuda_error() = e;
        return PJ_ERR_CUDA;
    }
    return s;
}

pj_status pj_inner_join_events(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws,
                               size_t ws_bytes, pj_stream stream, void* const* events)
{
    if (!valid_desc(d) || !out || !out->count || out->capacity < 0 || !events) return PJ_ERR_INVALID;
    if (out->capacity > 0 && (!out->build_row || !out->probe_row)) return PJ_ERR_INVALID;
    for (int i = 0; i < PJ_NUM_STAGES; ++i)
        if (!events[i]) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = resolve_plan(d, plan, &p);
    if (s != PJ_OK) return s;
    if ((s = check_inputs(d)) != PJ_OK) return s;
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    StageEvents E;
    E.ev = reinterpret_cast<cudaEvent_t*>(const_cast<void**>(events));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    if (d->key_bytes == 4)
        return run_join<int32_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st, E);
    return run_join<int64_t>(d, &p, L, w, out->build_row, out->probe_row, out->capacity, out->count, st, E);
}

pj_status pj_join_count(const pj_join_desc* d, const pj_plan* plan, int64_t* count_dev, void* ws, size_t ws_bytes,
                        pj_stream stream)
{
    if (!valid_desc(d) || !count_dev) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = resolve_plan(d, plan, &p);
    if (s != PJ_OK) return s;
    if ((s = check_inputs(d)) != PJ_OK) return s;
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    // capacity 0: the join kernel counts every match and writes none
    if (d->key_bytes == 4) return run_join<int32_t>(d, &p, L, w, nullptr, nullptr, 0, count_dev, st);
    return run_join<int64_t>(d, &p, L, w, nullptr, nullptr, 0, count_dev, st);
}

pj_status pj_check(void* ws, pj_stream stream)
{
    if (!ws) return PJ_ERR_WORKSPACE;
    PJ_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    uint32_t st = 0;
    PJ_CUDA(cudaMemcpy(&st, ws, sizeof(st), cudaMemcpyDeviceToHost));
    const uint32_t zero = 0;
    PJ_CUDA(cudaMemcpy(ws, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    if (st & ST_INTERNAL) return PJ_ERR_INTERNAL;
    if (st & ST_TIMEOUT) return PJ_ERR_TIMEOUT;
    if (st & ST_OVERFLOW) return PJ_ERR_OVERFLOW;
    if (st & ST_CAPACITY) return PJ_ERR_CAPACITY;
    return PJ_OK;
}

pj_status pj_hash_keys(const void* keys, int64_t n, int32_t key_bytes, uint32_t* out, pj_stream stream)
{
    if (n < 0 || (key_bytes != 4 && key_bytes != 8) || (n > 0 && (!keys || !out))) return PJ_ERR_INVALID;
    if (n == 0) return PJ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (key_bytes == 4)
        hash_keys_kernel<int32_t><<<grid_for(n, 256), 256, 0, st>>>(static_cast<const int32_t*>(keys), n, out);
    else
        hash_keys_kernel<int64_t><<<grid_for(n, 256), 256, 0, st>>>(static_cast<const int64_t*>(keys), n, out);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

pj_status pj_hash_slots(const void* keys, int64_t n, int32_t key_bytes, int32_t table_slots, int32_t slot_mode,
                        int32_t skip_bits, int32_t* out, pj_stream stream)
{
    if (n < 0 || (key_bytes != 4 && key_bytes != 8) || (n > 0 && (!keys || !out))) return PJ_ERR_INVALID;
    if (table_slots < 1 || (slot_mode != PJ_SLOT_FAST && slot_mode != PJ_SLOT_REF)) return PJ_ERR_INVALID;
    if (skip_bits < 0 || skip_bits > 31) return PJ_ERR_INVALID;
    if (n == 0) return PJ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int ref = slot_mode == PJ_SLOT_REF;
    if (key_bytes == 4)
        hash_slots_kernel<int32_t><<<grid_for(n, 256), 256, 0, st>>>(static_cast<const int32_t*>(keys), n,
                                                                    table_slots, ref, skip_bits, out);
    else
        hash_slots_kernel<int64_t><<<grid_for(n, 256), 256, 0, st>>>(static_cast<const int64_t*>(keys), n,
                                                                    table_slots, ref, skip_bits, out);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

pj_status pj_radix_histogram(const void* keys, int64_t n, int32_t key_bytes, int32_t digit_mode, int32_t bits1,
                             int32_t bits2, int32_t which, int32_t* hist, pj_stream stream)
{
    if (n < 0 || (key_bytes != 4 && key_bytes != 8) || !hist || (n > 0 && !keys)) return PJ_ERR_INVALID;
    if (digit_mode != PJ_DIGIT_RAW && digit_mode != PJ_DIGIT_HASH) return PJ_ERR_INVALID;
    if (bits1 < 0 || bits2 < 0 || bits1 + bits2 > 16 || which < 0 || which > 2) return PJ_ERR_INVALID;
    DigitFn f;
    int bits;
    if (which == 1) {
        f = digit_fn(digit_mode, 0, bits1, bits2);
        bits = bits1;
    } else if (which == 2) {
        f = digit_fn(digit_mode, bits1, bits2, 0);
        bits = bits2;
    } else {
        f = digit_fn(digit_mode, 0, bits1 + bits2, 0);
        bits = bits1 + bits2;
    }
    const int P = 1 << bits;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PJ_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * P, st));
    if (n == 0) return PJ_OK;
    const size_t smem = 4 * static_cast<size_t>(P);
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 4095) / 4096, sm_count() * 4)));
    if (key_bytes == 4) {
        PJ_CUDA(set_smem(global_hist_kernel<int32_t>, smem));
        global_hist_kernel<int32_t><<<grid, 512, smem, st>>>(static_cast<const int32_t*>(keys), n, f, P, hist);
    } else {
        PJ_CUDA(set_smem(global_hist_kernel<int64_t>, smem));
        global_hist_kernel<int64_t><<<grid, 512, smem, st>>>(static_cast<const int64_t*>(keys), n, f, P, hist);
    }
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

pj_status pj_partitioned_capacity(int64_t n, int32_t key_bytes, const pj_plan* plan, int64_t* tuples)
{
    if (n < 0 || n > INT32_MAX || (key_bytes != 4 && key_bytes != 8) || !plan || !tuples) return PJ_ERR_INVALID;
    *tuples = part_capacity(n, key_bytes, 1 << plan->bits1, scatter_items(plan));
    return PJ_OK;
}

pj_status pj_partition(const void* keys, int64_t n, int32_t key_bytes, const pj_plan* plan, void* tuples,
                       int64_t* offsets, void* ws, size_t ws_bytes, pj_stream stream)
{
    if (!plan || !tuples || !offsets || n < 0 || n > INT32_MAX || (key_bytes != 4 && key_bytes != 8) ||
        (n > 0 && !keys))
        return PJ_ERR_INVALID;
    pj_join_desc d{};
    d.build_keys = keys;
    d.probe_keys = keys;
    d.n_build = n;
    d.n_probe = 0;
    d.key_bytes = key_bytes;
    d.unique_build_keys = 1;
    pj_status s = check_plan(&d, plan);
    if (s != PJ_OK) return s;
    if (n > 0 && !aligned16(keys)) return PJ_ERR_ALIGNMENT;
    if (reinterpret_cast<uintptr_t>(tuples) & 15u) return PJ_ERR_ALIGNMENT;
    Layout L;
    if ((s = check_ws(&d, plan, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    uint32_t* status = reinterpret_cast<uint32_t*>(w + L.status);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(w + L.counters);
    PJ_CUDA(cudaMemsetAsync(w, 0, L.ctrl_end, st));
    const DigitFn f = digit_fn(plan->digit_mode, 0, plan->bits1, 0);
    if (key_bytes == 4)
        s = partition_side<int32_t>(static_cast<const int32_t*>(keys), n, L.b_chunk, L.b_items, f, L.P,
                                    reinterpret_cast<uint32_t*>(w + L.b_counts), reinterpret_cast<int32_t*>(w + L.b_tot),
                                    reinterpret_cast<int64_t*>(w + L.b_off), reinterpret_cast<uint64_t*>(w + L.b_tiles),
                                    ctr + CTR_BTILE, static_cast<uint32_t*>(tuples), L.b_cap, status, st);
    else
        s = partition_side<int64_t>(static_cast<const int64_t*>(keys), n, L.b_chunk, L.b_items, f, L.P,
                                    reinterpret_cast<uint32_t*>(w + L.b_counts), reinterpret_cast<int32_t*>(w + L.b_tot),
                                    reinterpret_cast<int64_t*>(w + L.b_off), reinterpret_cast<uint64_t*>(w + L.b_tiles),
                                    ctr + CTR_BTILE, static_cast<uint32_t*>(tuples), L.b_cap, status, st);
    if (s != PJ_OK) return s;
    partition_bounds_kernel<<<(L.P + 1 + 255) / 256, 256, 0, st>>>(reinterpret_cast<int64_t*>(w + L.b_off), L.b_items,
                                                                   L.P, offsets);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

pj_status pj_plan_exact(const pj_join_desc* d, void* ws, size_t ws_bytes, pj_plan* plan, pj_stream stream)
{
    if (!valid_desc(d) || !plan) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = pj_plan_default(d, &p);
    if (s != PJ_OK) return s;
    if (d->n_build == 0 || d->n_probe == 0) {
        *plan = p;
        return PJ_OK;
    }
    if ((s = check_inputs(d)) != PJ_OK) return s;
    // The histogram goes into the workspace's build-count area, which every
    // plan of this join has room for (P x items >= P).
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    const int P = 1 << p.bits1;
    int32_t* hist = reinterpret_cast<int32_t*>(static_cast<uint8_t*>(ws) + L.b_counts);
    if ((s = pj_radix_histogram(d->build_keys, d->n_build, d->key_bytes, p.digit_mode, p.bits1, 0, 0, hist, stream)) != PJ_OK)
        return s;
    int32_t* host = new int32_t[P];
    cudaError_t e = cudaMemcpyAsync(host, hist, sizeof(int32_t) * P, cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        delete[] host;
        last_cuda_error() = e;
        return PJ_ERR_CUDA;
    }
    int64_t mx = 0;
    for (int i = 0; i < P; ++i) mx = std::max<int64_t>(mx, host[i]);
    delete[] host;
    const int64_t cap = static_cast<int64_t>(p.table_slots * p.max_fill);
    // Hash splits cannot separate repeated keys: a partition beyond what
    // 2^MAX_SPLIT_LOG2 tables hold (duplicates) falls back to the
    // reference's position split.
    if (mx > cap * (int64_t(1) << MAX_SPLIT_LOG2) / 2) p.split_mode = PJ_SPLIT_POSITION;
    *plan = p;
    return PJ_OK;
}

}  // extern "C"
