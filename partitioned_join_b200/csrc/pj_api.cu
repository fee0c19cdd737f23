// pj_api.cu -- host side of the C ABI in include/pj.h: planning, workspace
// layout and the stage sequence (the reference's main.cu:762-892).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pj.h"
#include "pj_device.cuh"
#include "pj_internal.h"
#include "pj_join.cuh"
#include "pj_partition.cuh"

using namespace pj;
static_assert(MAX_HEAVY == PJ_MAX_HEAVY, "heavy-key capacity of the plan");

namespace {

// ---------------------------------------------------------------------------
// Fixed kernel configurations.
constexpr int SC_THREADS = 1024;
constexpr int SC_V32 = 4, SC_V64 = 2;  // keys per thread per round (one 16-byte vector)
#ifndef PJ_JOIN_THREADS
// 24 warps of up to 85 registers: the 1024-thread form (64 registers) spilled
// in the probe loop; 2^27 x 2^27 int32 join 2.43 -> 2.37 ms, 2^26 x 2^28
// int64 4.37 -> 3.73 ms (512, 640, 896 threads all measured slower; 832
// threads: int32 0.997 -> 1.007 ms, int64 1.95 -> 1.93 ms)
constexpr int JN_THREADS = 768;
#else
constexpr int JN_THREADS = PJ_JOIN_THREADS;
#endif
constexpr int MAX_SPLIT_LOG2 = 6;
constexpr int MAX_BUCKET_CAP = 65535;  // 16-bit bucket ends
constexpr int MAX_JOIN_CTAS_PER_SM = 4;
constexpr int HEAVY_SAMPLES = 1 << 16;     // probe keys the planner samples
constexpr int HEAVY_MIN_SAMPLES = 32;      // a heavy key holds >= 1/2048 of the sample
constexpr int64_t HEAVY_MIN_PROBE = 1 << 20;  // smaller probe sides: no heavy-key path
constexpr double HEAVY_MIN_SHARE = 0.5;       // share of the probe rows the heavy keys must hold
constexpr size_t LEARN_BYTES = 4096;          // features, activations and scores of the learned planner

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
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return DevInfo{};
    }
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && cache[dev].device == dev) return cache[dev];
    DevInfo d;
    d.device = dev;
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) d.sms = v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess)
        d.smem_optin = static_cast<size_t>(v);
    cudaGetLastError();
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

// Dynamic shared memory per CTA, less a reserve for static shared memory.
size_t smem_limit()
{
    const DevInfo d = dev_info();
    return (d.smem_optin > 0 ? d.smem_optin : 232448) - 1024;
}

int ilog2_floor(int64_t x)
{
    int b = 0;
    while ((int64_t(2) << b) <= x) ++b;
    return b;
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

int tuple_words(int key_bytes) { return key_bytes == 4 ? 2 : 4; }

// Shared memory of the scatter with P buffers of cap tuples each.
size_t scatter_smem(int key_bytes, int cap, int P)
{
    return static_cast<size_t>(P) * cap * tuple_words(key_bytes) * 4 + static_cast<size_t>(P) * 8;
}

// Tuples per partition buffer of a scatter whose rounds bring `round` tuples
// over P partitions, in groups of W: a round's expected arrivals per
// partition plus three standard deviations and one partial group, so that
// nearly every group completes inside the buffer and leaves as whole
// sectors; at most what shared memory holds beside `extra` bytes, at least W.
int wc_cap(int key_bytes, int W, int P, int round, size_t extra)
{
    const double m = static_cast<double>(round) / P;
    int want = static_cast<int>(std::ceil(m + 3.0 * std::sqrt(m))) + W;
    want = (want + W - 1) / W * W;
    const size_t room = smem_limit() > extra + static_cast<size_t>(P) * 8 ? smem_limit() - extra - static_cast<size_t>(P) * 8 : 0;
    const int fit = static_cast<int>(std::min<size_t>(room / (static_cast<size_t>(P) * tuple_words(key_bytes) * 4), 1 << 20)) / W * W;
    return std::max(W, std::min(want, fit));
}

bool valid_wc(int key_bytes, int W)
{
    if (W != 2 && W != 4 && W != 8 && W != 16 && W != 32) return false;
    return (W * tuple_words(key_bytes) * 4) % 16 == 0;
}

// Groups that are whole 32-byte sectors: the planner's choice.  Smaller
// groups are valid but leave sectors half written in L2 until a later
// flush, which measured at twice the DRAM traffic.
bool sector_wc(int key_bytes, int W) { return valid_wc(key_bytes, W) && (W * tuple_words(key_bytes) * 4) % 32 == 0; }

int bucket_nb_log2(int cap) { return std::max(1, ilog2_floor(std::max(2, cap / 2))); }

template <typename K>
size_t join_smem_k(int table_mode, int cap, int nb)
{
    switch (table_mode) {
    case PJ_TABLE_BUCKET: return JoinSmem<K, TABLE_BUCKET>::bytes(cap, nb);
    case PJ_TABLE_COMPACT: return JoinSmem<K, TABLE_COMPACT>::bytes(cap, nb);
    case PJ_TABLE_EXACT: return JoinSmem<K, TABLE_EXACT>::bytes(cap, nb);
    default: return JoinSmem<K, TABLE_OPEN>::bytes(cap, nb);
    }
}

// Shared memory of a join CTA for a table of cap tuples and 2^nb buckets
// (nb < 0: the default bucket count for cap).
size_t join_smem(int key_bytes, int table_mode, int cap, int nb = -1)
{
    if (nb < 0) nb = bucket_nb_log2(cap);
    return key_bytes == 4 ? join_smem_k<int32_t>(table_mode, cap, nb) : join_smem_k<int64_t>(table_mode, cap, nb);
}

// EXACT tables: an entry holds the build row in its low exact_row_bits
// bits and the hash bits above the bucket bits in the rest (8-byte keys:
// beside the key's low word).  With the partition's hash digits and the
// bucket they fix the whole MurmurHash3 value, which fixes a 4-byte key
// (a bijection) and, with the low word, an 8-byte key, so a lookup needs no
// build-tuple load.  That takes 2^nb buckets with
// digit bits + nb + (32 - row bits) >= 32.
int exact_row_bits(int64_t n_build)
{
    int r = 1;
    while (r < 31 && (int64_t(1) << r) < n_build) ++r;
    return r;
}

int plan_digit_bits(const pj_plan* p)
{
    return (p->digit_mode == PJ_DIGIT_HASH ? p->bits1 : 0) + (p->passes == 2 ? p->bits2 : 0);
}

// log2 of the bucket count of the plan's tables
int table_nb_log2(int64_t n_build, const pj_plan* p)
{
    const int nb = bucket_nb_log2(p->table_capacity);
    if (p->table_mode != PJ_TABLE_EXACT) return nb;
    return std::max(nb, exact_row_bits(n_build) - plan_digit_bits(p));
}

// Largest EXACT capacity (a multiple of 128 tuples) with at least 2^nb_min
// buckets; 0 if none fits shared memory.
int exact_table_capacity(int key_bytes, int nb_min)
{
    if (nb_min > 20) return 0;
    int best = 0;
    for (int cap = 128; cap <= MAX_BUCKET_CAP; cap += 128)
        if (join_smem(key_bytes, PJ_TABLE_EXACT, cap, std::max(bucket_nb_log2(cap), nb_min)) <= smem_limit()) best = cap;
    return best;
}

int max_table_capacity(int key_bytes, int table_mode)
{
    int lo = 64, hi = table_mode == PJ_TABLE_OPEN ? (1 << 20) : MAX_BUCKET_CAP;
    const size_t lim = smem_limit();
    if (join_smem(key_bytes, table_mode, lo) > lim) return 0;
    while (lo < hi) {  // largest cap that fits
        const int mid = lo + (hi - lo + 1) / 2;
        if (join_smem(key_bytes, table_mode, mid) <= lim) lo = mid; else hi = mid - 1;
    }
    return lo & ~127;
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

int pass2_wc(int key_bytes, const pj_plan* p);

pj_status check_plan(const pj_join_desc* d, const pj_plan* p)
{
    if (p->passes != 1 && p->passes != 2) return PJ_ERR_INVALID;
    if (p->passes == 1 ? p->bits2 != 0 : (p->bits1 < 1 || p->bits2 < 1 || p->bits1 + p->bits2 > 22))
        return PJ_ERR_INVALID;
    if (p->passes == 2 && pass2_wc(d->key_bytes, p) == 0) return PJ_ERR_INVALID;
    if (p->bits1 < 0 || p->bits1 > 16) return PJ_ERR_INVALID;
    if (!valid_wc(d->key_bytes, p->wc_tuples)) return PJ_ERR_INVALID;
    if (scatter_smem(d->key_bytes, p->wc_tuples, 1 << p->bits1) > smem_limit()) return PJ_ERR_INVALID;
    if (p->digit_mode != PJ_DIGIT_RAW && p->digit_mode != PJ_DIGIT_HASH) return PJ_ERR_INVALID;
    if (p->table_mode != PJ_TABLE_BUCKET && p->table_mode != PJ_TABLE_OPEN && p->table_mode != PJ_TABLE_COMPACT &&
        p->table_mode != PJ_TABLE_EXACT)
        return PJ_ERR_INVALID;
    if (p->slot_mode != PJ_SLOT_FAST && p->slot_mode != PJ_SLOT_REF) return PJ_ERR_INVALID;
    if (p->split_mode != PJ_SPLIT_HASH && p->split_mode != PJ_SPLIT_POSITION) return PJ_ERR_INVALID;
    if (p->table_mode == PJ_TABLE_EXACT) {
        if (p->table_capacity < 64 || p->table_capacity > MAX_BUCKET_CAP) return PJ_ERR_INVALID;
        const int nb = table_nb_log2(d->n_build, p);
        if (nb > 20 || join_smem(d->key_bytes, PJ_TABLE_EXACT, p->table_capacity, nb) > smem_limit())
            return PJ_ERR_INVALID;
    } else if (p->table_capacity < 64 || p->table_capacity > max_table_capacity(d->key_bytes, p->table_mode)) {
        return PJ_ERR_INVALID;
    }
    if (p->probe_chunk < 16 || (p->probe_chunk & 15)) return PJ_ERR_INVALID;
    if (p->scatter_ctas_per_sm < 1 || p->scatter_ctas_per_sm > 8) return PJ_ERR_INVALID;
    if (p->hist_split < 1 || p->hist_split > 16) return PJ_ERR_INVALID;
    if (p->table_mode == PJ_TABLE_OPEN && !(p->max_fill > 0.05f && p->max_fill <= 0.95f)) return PJ_ERR_INVALID;
    if (p->n_heavy < 0 || p->n_heavy > PJ_MAX_HEAVY) return PJ_ERR_INVALID;
    if (p->n_heavy > 0 && scatter_smem(d->key_bytes, p->wc_tuples, 1 << p->bits1) + HeavyTable::BYTES + 16 > smem_limit())
        return PJ_ERR_INVALID;  // the probe scatter also holds the heavy table
    // hash bits: digits + hash split + bucket/slot bits must fit 32
    const int digit_bits = plan_digit_bits(p);
    const int slot_bits = p->table_mode != PJ_TABLE_OPEN ? table_nb_log2(d->n_build, p) : 12;
    // digits and bucket bits disjoint; the bits of a hash split (below the
    // digits) may overlap the bucket bits: pieces stay exact, buckets coarser
    if (digit_bits + slot_bits > 32 || digit_bits + MAX_SPLIT_LOG2 > 31) return PJ_ERR_INVALID;
    return PJ_OK;
}

// Write-combining group (tuples): the smallest whole-sector group whose
// buffers fit shared memory at a fan-out of 2^b partitions; 0 if none fits.
// Where the fan-out is low the buffers hold several groups (wc_cap).
int pick_wc(int key_bytes, int b)
{
    for (int W : {2, 4, 8, 16, 32})
        if (sector_wc(key_bytes, W) && scatter_smem(key_bytes, W, 1 << b) <= smem_limit()) return W;
    return 0;
}

// Write-combining width of a two-pass plan's second pass (its own fan-out).
int pass2_wc(int key_bytes, const pj_plan* p) { return pick_wc(key_bytes, p->bits2); }

// Fewest radix bits whose expected build partition fills at most 7/8 of a
// table of cap tuples.
int bits_for_table(int64_t n_build, int64_t cap)
{
    const int64_t target = std::max<int64_t>(1, cap - cap / 8);
    return ilog2_ceil(std::max<int64_t>(1, (n_build + target - 1) / target));
}

// Heavy probe keys of a key sample: those seen at least min_count times
// (the most frequent PJ_MAX_HEAVY of them) go to plan->heavy_keys; returns
// the share of the sample they cover.
double heavy_from_sample(const std::vector<int64_t>& keys, int min_count, pj_plan* plan)
{
    // Key frequencies in an open-addressing table (linear probing, at most
    // half full): a planning call counts up to 65 536 sampled keys, and a
    // node-based hash map took milliseconds for that.
    size_t cap = 16;
    while (cap < 2 * keys.size()) cap <<= 1;
    std::vector<int64_t> slot_key(cap);
    std::vector<int32_t> slot_count(cap, 0);  // 0: empty
    for (int64_t k : keys) {
        uint64_t x = static_cast<uint64_t>(k);  // splitmix64 finaliser as the table's hash
        x ^= x >> 30;
        x *= 0xbf58476d1ce4e5b9ull;
        x ^= x >> 27;
        x *= 0x94d049bb133111ebull;
        x ^= x >> 31;
        size_t i = static_cast<size_t>(x) & (cap - 1);
        while (slot_count[i] != 0 && slot_key[i] != k) i = (i + 1) & (cap - 1);
        slot_key[i] = k;
        ++slot_count[i];
    }
    std::vector<std::pair<int, int64_t>> heavy;
    for (size_t i = 0; i < cap; ++i)
        if (slot_count[i] >= min_count) heavy.emplace_back(slot_count[i], slot_key[i]);
    std::sort(heavy.begin(), heavy.end(), [](const auto& x, const auto& y) {
        return x.first != y.first ? x.first > y.first : x.second < y.second;
    });
    plan->n_heavy = static_cast<int32_t>(std::min<size_t>(heavy.size(), PJ_MAX_HEAVY));
    int64_t covered = 0;
    for (int i = 0; i < plan->n_heavy; ++i) {
        plan->heavy_keys[i] = heavy[i].second;
        covered += heavy[i].first;
    }
    return keys.empty() ? 0.0 : static_cast<double>(covered) / static_cast<double>(keys.size());
}

// Resident join CTAs per SM for this plan: shared memory and threads bound it.
int join_ctas_per_sm(int key_bytes, const pj_plan* p)
{
    const size_t smem = join_smem(key_bytes, p->table_mode, p->table_capacity);
    const int by_smem = static_cast<int>((smem_limit() + 1024) / std::max<size_t>(smem + 1024, 1));
    const int by_threads = 2048 / JN_THREADS;
    return std::max(1, std::min({MAX_JOIN_CTAS_PER_SM, by_smem, by_threads}));
}

// Build tuples one table holds.
int table_tuples(const pj_plan* p)
{
    return p->table_mode != PJ_TABLE_OPEN ? p->table_capacity
                                          : std::max(1, static_cast<int>(p->table_capacity * p->max_fill));
}

// ---------------------------------------------------------------------------
// Workspace layout.  Everything 256-byte aligned.
struct Layout {
    int P = 1;    // partitions the join sees (P1 * P2 for two-pass plans)
    int P1 = 1;   // partitions of the first pass
    int C = 0;    // two-pass plans: slices per first-pass partition in the second pass
    int64_t b_cap2 = 0, p_cap2 = 0;  // tuples of the second pass's output
    size_t b_tiles2 = 0, p_tiles2 = 0, b_counts2 = 0, p_counts2 = 0, b_off2 = 0, p_off2 = 0;
    size_t b_tuples2 = 0, p_tuples2 = 0;
    int64_t b_tiles2_n = 0, p_tiles2_n = 0;
    int b_items = 1, p_items = 1;
    int64_t b_chunk = 16, p_chunk = 16;
    int64_t b_cap = 0, p_cap = 0;  // tuples
    int64_t max_items = 0;
    size_t status = 0, counters = 0, b_tiles = 0, p_tiles = 0, i_tiles = 0, b_tot = 0, p_tot = 0;
    size_t b_counts = 0, p_counts = 0, heavy_total = 0, heavy_items = 0, ctrl_end = 0;
    size_t heavy_row = 0, sample = 0, learn = 0;
    size_t b_off = 0, p_off = 0, split = 0, items = 0, item_off = 0, item_part = 0;
    size_t cta_q = 0, cta_last = 0, seg = 0, over_b = 0, over_p = 0;
    int max_ctas = 0;
    int64_t over_cap = 0;
    size_t b_tuples = 0, p_tuples = 0, total = 0;
    int64_t b_tiles_n = 0, p_tiles_n = 0, i_tiles_n = 0;
};

constexpr int CTR_QUEUE = 0, CTR_BTILE = 1, CTR_PTILE = 2, CTR_ITILE = 3, CTR_BTILE2 = 4, CTR_PTILE2 = 5;

int64_t chunk_for(int64_t n, int items)
{
    int64_t c = (n + items - 1) / std::max(items, 1);
    c = (c + 15) / 16 * 16;
    return std::max<int64_t>(c, 16);
}

int scatter_items(const pj_plan* p) { return sm_count() * std::max(1, p->scatter_ctas_per_sm); }

int64_t part_capacity(int64_t n, int P, int items, int W) { return n + static_cast<int64_t>(items) * P * (W - 1) + W; }

Layout make_layout(const pj_join_desc* d, const pj_plan* p)
{
    Layout L;
    const bool two = p->passes == 2;
    L.P1 = 1 << p->bits1;
    L.P = two ? L.P1 << p->bits2 : L.P1;
    L.b_items = L.p_items = scatter_items(p);
    L.b_chunk = chunk_for(d->n_build, L.b_items);
    L.p_chunk = chunk_for(d->n_probe, L.p_items);
    L.b_cap = part_capacity(d->n_build, L.P1, L.b_items, p->wc_tuples);
    L.p_cap = part_capacity(d->n_probe, L.P1, L.p_items, p->wc_tuples);
    if (two) {
        // second pass: about four items per SM over the first pass's
        // partitions (items of one partition's slices are near-equal)
        L.C = std::max(1, (4 * sm_count() + L.P1 - 1) / L.P1);
        L.b_cap2 = part_capacity(d->n_build, L.P, L.C, pass2_wc(d->key_bytes, p));
        L.p_cap2 = part_capacity(d->n_probe, L.P, L.C, pass2_wc(d->key_bytes, p));
    }
    const int64_t m2 = static_cast<int64_t>(L.P) * L.C;  // second-pass segments per side
    L.b_tiles2_n = L.p_tiles2_n = two ? (m2 + SCAN_TILE - 1) / SCAN_TILE + 1 : 0;
    const int64_t mb = static_cast<int64_t>(L.P1) * L.b_items, mp = static_cast<int64_t>(L.P1) * L.p_items;
    L.b_tiles_n = (mb + SCAN_TILE - 1) / SCAN_TILE + 1;
    L.p_tiles_n = (mp + SCAN_TILE - 1) / SCAN_TILE + 1;
    L.i_tiles_n = (L.P + SCAN_TILE - 1) / SCAN_TILE + 1;
    // items: per partition at most 2^MAX_SPLIT_LOG2 hash pieces, or
    // table-sized position pieces, times ceil(probe range / probe_chunk)
    const int64_t per_piece = std::max<int64_t>(16, table_tuples(p) / 16 * 16);
    const int64_t max_pieces = std::max<int64_t>(static_cast<int64_t>(L.P) << MAX_SPLIT_LOG2, L.P + L.b_cap / per_piece);
    const int64_t max_chunks = L.P + L.p_cap / p->probe_chunk + 1;
    L.max_items = std::min<int64_t>(max_pieces * max_chunks, static_cast<int64_t>(L.P) * 4096 + max_pieces + max_chunks);
    L.max_items = std::min<int64_t>(L.max_items, int64_t(1) << 30);
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = align_up(o + bytes, 256); return at; };
    // control block, zeroed at the start of every call
    L.status = take(4);
    L.counters = take(4 * 8);
    L.b_tiles = take(8 * L.b_tiles_n);
    L.p_tiles = take(8 * L.p_tiles_n);
    L.i_tiles = take(8 * L.i_tiles_n);
    L.b_tot = take(4 * static_cast<size_t>(L.P));
    L.p_tot = take(4 * static_cast<size_t>(L.P));
    L.b_counts = take(4 * static_cast<size_t>(mb));
    L.p_counts = take(4 * static_cast<size_t>(mp));
    L.heavy_total = take(8);
    L.heavy_items = take(8 * static_cast<size_t>(L.p_items));
    if (two) {
        L.b_tiles2 = take(8 * L.b_tiles2_n);
        L.p_tiles2 = take(8 * L.p_tiles2_n);
        L.b_counts2 = take(4 * static_cast<size_t>(m2));
        L.p_counts2 = take(4 * static_cast<size_t>(m2));
    }
    L.ctrl_end = o;
    L.heavy_row = take(4 * MAX_HEAVY);
    L.sample = take(8 * static_cast<size_t>(HEAVY_SAMPLES));
    L.learn = take(LEARN_BYTES);
    L.b_off = take(8 * static_cast<size_t>(mb + 1));
    L.p_off = take(8 * static_cast<size_t>(mp + 1));
    L.split = take(4 * static_cast<size_t>(L.P));
    L.items = take(8 * static_cast<size_t>(L.P));
    L.item_off = take(8 * static_cast<size_t>(L.P + 1));
    L.item_part = take(4 * static_cast<size_t>(L.max_items));
    // output fix-up: per join CTA records, segments, and room for the
    // reserved positions past the caller's capacity (one chunk per CTA)
    // the fix-up plan kernel records one gap per join CTA in a 1024-thread block
    L.max_ctas = std::min(sm_count() * join_ctas_per_sm(d->key_bytes, p), MAX_FIXUP_CTAS);
    L.over_cap = static_cast<int64_t>(L.max_ctas) * OUT_CHUNK;
    L.cta_q = take(8 * static_cast<size_t>(L.max_ctas));
    L.cta_last = take(8 * static_cast<size_t>(L.max_ctas));
    L.seg = take(8 * (4 + 4 * static_cast<size_t>(L.max_ctas + 2)));
    L.over_b = take(4 * static_cast<size_t>(L.over_cap));
    L.over_p = take(4 * static_cast<size_t>(L.over_cap));
    const int TW = tuple_words(d->key_bytes);
    L.b_tuples = take(4 * static_cast<size_t>(TW) * L.b_cap + 64);
    L.p_tuples = take(4 * static_cast<size_t>(TW) * L.p_cap + 64);
    if (two) {
        L.b_off2 = take(8 * static_cast<size_t>(m2 + 1));
        L.p_off2 = take(8 * static_cast<size_t>(m2 + 1));
        L.b_tuples2 = take(4 * static_cast<size_t>(TW) * L.b_cap2 + 64);
        L.p_tuples2 = take(4 * static_cast<size_t>(TW) * L.p_cap2 + 64);
    }
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

cudaError_t& last_cuda_error()
{
    static thread_local cudaError_t e = cudaSuccess;
    return e;
}

#define PJ_CUDA(call)                                            \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) {                                 \
            last_cuda_error() = e_;                              \
            return PJ_ERR_CUDA;                                  \
        }                                                        \
    } while (0)

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

// Features of the learned planner, from a sample of the probe keys (one
// CTA): a 1024-bin sketch of the sample by hash, sorted by count, read at
// log-spaced ranks (the shape of the key-frequency curve, whichever keys are
// heavy), plus the sizes and the key width.  The sample keys go to
// sample_out for the heavy-key candidates.
constexpr int SKETCH_BINS = 1024;
__constant__ int c_feature_ranks[20] = {0, 1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768};

template <typename K>
__global__ void __launch_bounds__(SKETCH_BINS) plan_features_kernel(const K* __restrict__ keys, int64_t n,
                                                                   int32_t samples, int64_t* __restrict__ sample_out,
                                                                   float* __restrict__ feat, float log_nb, float log_np,
                                                                   float key_bytes, float unique)
{
    __shared__ uint32_t bins[SKETCH_BINS];
    const int t = threadIdx.x;
    bins[t] = 0;
    __syncthreads();
    for (int s = t; s < samples; s += SKETCH_BINS) {
        const K k = keys[sample_pos(s, n)];
        sample_out[s] = static_cast<int64_t>(k);
        atomicAdd(&bins[hash_key(k) & (SKETCH_BINS - 1)], 1u);
    }
    __syncthreads();
    // bitonic sort, descending
    for (int size = 2; size <= SKETCH_BINS; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int o = t ^ stride;
            if (o > t) {
                const uint32_t a = bins[t], b = bins[o];
                const bool desc = (t & size) == 0;
                if (desc ? a < b : a > b) {
                    bins[t] = b;
                    bins[o] = a;
                }
            }
            __syncthreads();
        }
    const float scale = static_cast<float>(SKETCH_BINS) / static_cast<float>(samples > 0 ? samples : 1);
    if (t < 20) feat[t] = log2f(1.0f + bins[c_feature_ranks[t]] * scale);
    if (t == 0) {
        uint32_t top = 0, nonempty = 0;
        for (int i = 0; i < 16; ++i) top += bins[i];
        for (int i = 0; i < SKETCH_BINS; ++i) nonempty += bins[i] ? 1u : 0u;
        feat[20] = static_cast<float>(top) / static_cast<float>(samples > 0 ? samples : 1);
        feat[21] = static_cast<float>(nonempty) / SKETCH_BINS;
        feat[22] = log_nb / 32.0f;
        feat[23] = log_np / 32.0f;
        feat[24] = (log_np - log_nb) / 8.0f;
        feat[25] = key_bytes / 8.0f;
        feat[26] = unique;
        for (int i = 27; i < PJ_MLP_FEATURES; ++i) feat[i] = 0.0f;
    }
}

// Payload materialisation after the join: dst[i] = src[row[i]] for the
// count entries written (the step after the join in a query engine; the
// reference emits the probe payload inside its join record instead,
// hash_join_kernels.cuh:155-163).  Either side may be absent.
template <typename T>
__global__ void gather_payload_kernel(const int32_t* __restrict__ build_row, const int32_t* __restrict__ probe_row,
                                      const T* __restrict__ build_src, const T* __restrict__ probe_src,
                                      T* __restrict__ build_dst, T* __restrict__ probe_dst,
                                      const unsigned long long* __restrict__ count, int64_t capacity)
{
    const long long n = static_cast<long long>(*count) < capacity ? static_cast<long long>(*count) : capacity;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (build_dst) build_dst[i] = build_src[build_row[i]];
        if (probe_dst) probe_dst[i] = probe_src[probe_row[i]];
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

// Heavy probe keys of one join: the set and where their pairs go.
struct HeavyCtx {
    const HeavySet* hs = nullptr;  // nullptr: no heavy path
    HeavyOut out{};
};

template <typename K, bool HASHD, bool HEAVY>
pj_status launch_hist_t(const K* keys, int64_t n, int64_t chunk, int items, int hsplit, DigitFn f, int P,
                        uint32_t* counts, int32_t* totals, const HeavyCtx& hc, cudaStream_t st)
{
    const size_t smem = 4 * static_cast<size_t>((P + 3) & ~3) + (HEAVY ? HeavyTable::BYTES : 0);
    auto* kern = hist_keys_kernel<K, HASHD, HEAVY>;
    PJ_CUDA(set_smem(kern, smem));
    typename HeavyArg<HEAVY>::type h{};
    if constexpr (HEAVY) h = *hc.hs;
    kern<<<items * hsplit, HIST_THREADS, smem, st>>>(keys, n, chunk, items, hsplit, f, P, counts, totals, h, hc.out);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

// hc.hs: heavy probe keys to leave out (nullptr: none)
template <typename K>
pj_status launch_hist(const K* keys, int64_t n, int64_t chunk, int items, int hsplit, DigitFn f, int P,
                      uint32_t* counts, int32_t* totals, cudaStream_t st, const HeavyCtx& hc = HeavyCtx())
{
    const bool hd = f.mode == PJ_DIGIT_HASH;
    if (hc.hs)
        return hd ? launch_hist_t<K, true, true>(keys, n, chunk, items, hsplit, f, P, counts, totals, hc, st)
                  : launch_hist_t<K, false, true>(keys, n, chunk, items, hsplit, f, P, counts, totals, hc, st);
    return hd ? launch_hist_t<K, true, false>(keys, n, chunk, items, hsplit, f, P, counts, totals, hc, st)
              : launch_hist_t<K, false, false>(keys, n, chunk, items, hsplit, f, P, counts, totals, hc, st);
}

template <typename TIn>
pj_status launch_scan(const TIn* in, int64_t m, uint32_t round_to, int64_t* out, uint64_t* tiles,
                      uint32_t* tile_counter, uint32_t* status, cudaStream_t st,
                      ScanWait wait = ScanWait{-1, SPIN_LIMIT})
{
    const int64_t ntiles = std::max<int64_t>(1, (m + SCAN_TILE - 1) / SCAN_TILE);
    lookback_scan_kernel<TIn><<<static_cast<unsigned>(ntiles), SCAN_THREADS, 0, st>>>(in, m, round_to, out, tiles,
                                                                                    tile_counter, status, wait);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K, int W, bool HASHD, bool HEAVY>
pj_status launch_scatter_t(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P,
                           const int64_t* offsets, uint32_t* out, int64_t out_cap, uint32_t* status,
                           const HeavyCtx& hc, cudaStream_t st)
{
    auto* kern = scatter_keys_kernel<K, SC_THREADS, sc_v<K>(), W, HASHD, HEAVY>;
    constexpr int TW = WcTraits<K, W>::TW;
    const int cap = wc_cap(sizeof(K), W, P, SC_THREADS * sc_v<K>(), HEAVY ? HeavyTable::BYTES + 16 : 0);
    const size_t smem = HEAVY ? heavy_table_offset(P, cap * TW) + HeavyTable::BYTES : scatter_smem(sizeof(K), cap, P);
    PJ_CUDA(set_smem(kern, smem));
    typename HeavyArg<HEAVY>::type h{};
    if constexpr (HEAVY) h = *hc.hs;
    kern<<<items, SC_THREADS, smem, st>>>(keys, n, chunk, items, f, P, cap, offsets, out,
                                         static_cast<uint32_t>(std::min<int64_t>(out_cap, UINT32_MAX)), status, h,
                                         hc.out);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K, int W>
pj_status launch_scatter_w(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P,
                           const int64_t* offsets, uint32_t* out, int64_t out_cap, uint32_t* status,
                           const HeavyCtx& hc, cudaStream_t st)
{
    const bool hd = f.mode == PJ_DIGIT_HASH;
    if (hc.hs)
        return hd ? launch_scatter_t<K, W, true, true>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st)
                  : launch_scatter_t<K, W, false, true>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    return hd ? launch_scatter_t<K, W, true, false>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st)
              : launch_scatter_t<K, W, false, false>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
}

template <typename K>
pj_status launch_scatter(const K* keys, int64_t n, int64_t chunk, int items, DigitFn f, int P, int W,
                         const int64_t* offsets, uint32_t* out, int64_t out_cap, uint32_t* status, cudaStream_t st,
                         const HeavyCtx& hc = HeavyCtx())
{
    if (W == 2) return launch_scatter_w<K, 2>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    if (W == 4) return launch_scatter_w<K, 4>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    if (W == 8) return launch_scatter_w<K, 8>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    if (W == 16) return launch_scatter_w<K, 16>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    if (W == 32) return launch_scatter_w<K, 32>(keys, n, chunk, items, f, P, offsets, out, out_cap, status, hc, st);
    return PJ_ERR_INVALID;
}

template <typename K, int TABLE, bool UNIQUE, bool HASH_SPLIT, bool SLOT_REF>
pj_status launch_join_t(const JoinArgs& a, cudaStream_t st)
{
    auto* kern = join_kernel<K, TABLE, UNIQUE, HASH_SPLIT, SLOT_REF, JN_THREADS>;
    const size_t smem = JoinSmem<K, TABLE>::bytes(a.cap, a.nb_log2);
    PJ_CUDA(set_smem(kern, smem));
    int per_sm = 0;
    PJ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, JN_THREADS, smem));
    per_sm = std::min(std::max(per_sm, 1), MAX_JOIN_CTAS_PER_SM);
    const int grid = std::min(sm_count() * per_sm, a.max_ctas);
    kern<<<grid, JN_THREADS, smem, st>>>(a);
    PJ_CUDA(cudaGetLastError());
    // fix-up: dense output and the true count
    const int fix_threads = std::min(MAX_FIXUP_CTAS, (grid + 31) / 32 * 32);
    join_fixup_plan_kernel<<<1, fix_threads, 0, st>>>(a.cta_q, a.cta_last, grid, a.count, a.base_count, a.capacity,
                                               a.out_build != nullptr ? 1 : 0, a.seg, a.status);
    PJ_CUDA(cudaGetLastError());
    if (a.out_build != nullptr) {
        join_fixup_move_kernel<<<sm_count() * 2, 512, 0, st>>>(a.seg, grid, a.out_build, a.out_probe, a.capacity,
                                                               a.over_build, a.over_probe);
        PJ_CUDA(cudaGetLastError());
    }
    return PJ_OK;
}

template <typename K, int TABLE>
pj_status launch_join_tab(const JoinArgs& a, bool unique, bool hash_split, bool slot_ref, cudaStream_t st)
{
    if (unique) {
        if (hash_split)
            return slot_ref ? launch_join_t<K, TABLE, true, true, true>(a, st)
                            : launch_join_t<K, TABLE, true, true, false>(a, st);
        return slot_ref ? launch_join_t<K, TABLE, true, false, true>(a, st)
                        : launch_join_t<K, TABLE, true, false, false>(a, st);
    }
    if (hash_split)
        return slot_ref ? launch_join_t<K, TABLE, false, true, true>(a, st)
                        : launch_join_t<K, TABLE, false, true, false>(a, st);
    return slot_ref ? launch_join_t<K, TABLE, false, false, true>(a, st)
                    : launch_join_t<K, TABLE, false, false, false>(a, st);
}

template <typename K>
pj_status launch_join(const JoinArgs& a, int table_mode, bool unique, bool hash_split, bool slot_ref, cudaStream_t st)
{
    if (table_mode == PJ_TABLE_BUCKET) return launch_join_tab<K, TABLE_BUCKET>(a, unique, hash_split, false, st);
    if (table_mode == PJ_TABLE_COMPACT) return launch_join_tab<K, TABLE_COMPACT>(a, unique, hash_split, false, st);
    if (table_mode == PJ_TABLE_EXACT) return launch_join_tab<K, TABLE_EXACT>(a, unique, hash_split, false, st);
    return launch_join_tab<K, TABLE_OPEN>(a, unique, hash_split, slot_ref, st);
}

// Optional stage events: ev[i] is recorded before stage i, ev[PJ_STAGE_TOTAL] at the end.
struct StageEvents {
    cudaEvent_t* ev = nullptr;
    void mark(int i, cudaStream_t st) const
    {
        if (ev) cudaEventRecord(ev[i], st);
    }
};

// Partition one column: histogram -> look-back scan -> scatter.
template <typename K>
pj_status partition_column(const K* keys, int64_t n, const pj_plan* p, const Layout& L, int side, uint8_t* ws,
                           uint32_t* tuples, int64_t cap, const StageEvents& E, int stage0, cudaStream_t st,
                           const HeavyCtx& hc = HeavyCtx())
{
    const DigitFn f = digit_fn(p->digit_mode, 0, p->bits1, 0);
    const int P1 = L.P1;
    const int64_t chunk = side == 0 ? L.b_chunk : L.p_chunk;
    const int items = side == 0 ? L.b_items : L.p_items;
    uint32_t* status = reinterpret_cast<uint32_t*>(ws + L.status);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(ws + L.counters);
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + (side == 0 ? L.b_counts : L.p_counts));
    // per-partition totals feed the join's work split: the second pass
    // writes them for two-pass plans
    int32_t* tot = p->passes == 2 ? nullptr : reinterpret_cast<int32_t*>(ws + (side == 0 ? L.b_tot : L.p_tot));
    int64_t* off = reinterpret_cast<int64_t*>(ws + (side == 0 ? L.b_off : L.p_off));
    uint64_t* tiles = reinterpret_cast<uint64_t*>(ws + (side == 0 ? L.b_tiles : L.p_tiles));
    pj_status s;
    E.mark(stage0, st);
    if ((s = launch_hist<K>(keys, n, chunk, items, p->hist_split, f, P1, counts, tot, st, hc)) != PJ_OK) return s;
    E.mark(stage0 + 1, st);
    if ((s = launch_scan<uint32_t>(counts, static_cast<int64_t>(P1) * items, static_cast<uint32_t>(p->wc_tuples), off,
                                   tiles, ctr + (side == 0 ? CTR_BTILE : CTR_PTILE), status, st)) != PJ_OK)
        return s;
    E.mark(stage0 + 2, st);
    return launch_scatter<K>(keys, n, chunk, items, f, P1, p->wc_tuples, off, tuples, cap, status, st, hc);
}

// Second pass of a two-pass plan over one side's first-pass tuples:
// histogram -> look-back scan -> scatter into the side's second tuple buffer.
// The digit is the next bits2 hash bits below those the first pass used.
template <typename K, int W>
pj_status launch_scatter_tuples(const uint32_t* in, const Pass2Items& it, int n_items, DigitFn f, int P2,
                                const int64_t* off, uint32_t* out, int64_t cap, uint32_t* status, cudaStream_t st)
{
    constexpr int VT = sizeof(K) == 4 ? 4 : 2;
    auto* kern = scatter_tuples_kernel<K, SC_THREADS, VT, W>;
    const int bcap = wc_cap(sizeof(K), W, P2, SC_THREADS * VT, 0);
    const size_t smem = scatter_smem(sizeof(K), bcap, P2);
    PJ_CUDA(set_smem(kern, smem));
    const int grid = std::min(n_items, sm_count());
    kern<<<grid, SC_THREADS, smem, st>>>(in, it, n_items, f, P2, bcap, off,
                                        out, static_cast<uint32_t>(std::min<int64_t>(cap, UINT32_MAX)), status);
    PJ_CUDA(cudaGetLastError());
    return PJ_OK;
}

template <typename K>
pj_status partition_pass2(const pj_plan* p, const Layout& L, int side, uint8_t* ws, uint32_t* out, int64_t cap,
                          cudaStream_t st)
{
    const int hb = p->digit_mode == PJ_DIGIT_HASH ? p->bits1 : 0;  // hash bits the first pass used
    const DigitFn f = digit_fn(PJ_DIGIT_HASH, hb, p->bits2, 0);
    const int P2 = 1 << p->bits2;
    const int items1 = side == 0 ? L.b_items : L.p_items;
    const int n_items = L.P1 * L.C;
    uint32_t* status = reinterpret_cast<uint32_t*>(ws + L.status);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(ws + L.counters);
    const Pass2Items it{reinterpret_cast<const int64_t*>(ws + (side == 0 ? L.b_off : L.p_off)), items1, L.C};
    const uint32_t* in = reinterpret_cast<const uint32_t*>(ws + (side == 0 ? L.b_tuples : L.p_tuples));
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + (side == 0 ? L.b_counts2 : L.p_counts2));
    int32_t* tot = reinterpret_cast<int32_t*>(ws + (side == 0 ? L.b_tot : L.p_tot));
    int64_t* off = reinterpret_cast<int64_t*>(ws + (side == 0 ? L.b_off2 : L.p_off2));
    uint64_t* tiles = reinterpret_cast<uint64_t*>(ws + (side == 0 ? L.b_tiles2 : L.p_tiles2));
    const size_t hsmem = 4 * static_cast<size_t>(P2);
    PJ_CUDA(set_smem(hist_tuples_kernel<K>, hsmem));
    hist_tuples_kernel<K><<<n_items * p->hist_split, HIST_THREADS, hsmem, st>>>(in, it, n_items, p->hist_split, f, P2,
                                                                               L.P1, counts, tot);
    PJ_CUDA(cudaGetLastError());
    pj_status s;
    const int W2 = pass2_wc(static_cast<int>(sizeof(K)), p);
    if ((s = launch_scan<uint32_t>(counts, static_cast<int64_t>(P2) * n_items, static_cast<uint32_t>(W2), off, tiles,
                                   ctr + (side == 0 ? CTR_BTILE2 : CTR_PTILE2), status, st)) != PJ_OK)
        return s;
    switch (W2) {
    case 2: return launch_scatter_tuples<K, 2>(in, it, n_items, f, P2, off, out, cap, status, st);
    case 4: return launch_scatter_tuples<K, 4>(in, it, n_items, f, P2, off, out, cap, status, st);
    case 8: return launch_scatter_tuples<K, 8>(in, it, n_items, f, P2, off, out, cap, status, st);
    case 16: return launch_scatter_tuples<K, 16>(in, it, n_items, f, P2, off, out, cap, status, st);
    case 32: return launch_scatter_tuples<K, 32>(in, it, n_items, f, P2, off, out, cap, status, st);
    default: return PJ_ERR_INVALID;
    }
}

template <typename K>
pj_status run_join(const pj_join_desc* d, const pj_plan* p, const Layout& L, uint8_t* ws, int32_t* out_b,
                   int32_t* out_p, int64_t capacity, int64_t* count, void* pay_b, void* pay_p, cudaStream_t st,
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
    pj_status s;
    // heavy-key path: unique build keys and a plan that names heavy probe keys
    HeavySet hs{};
    HeavyCtx hc;
    auto* heavy_total = reinterpret_cast<unsigned long long*>(ws + L.heavy_total);
    if (p->n_heavy > 0 && d->unique_build_keys) {
        hs.n = p->n_heavy;
        for (int i = 0; i < p->n_heavy; ++i) hs.keys[i] = p->heavy_keys[i];
        int32_t* hrow = reinterpret_cast<int32_t*>(ws + L.heavy_row);
        PJ_CUDA(cudaMemsetAsync(hrow, 0xff, 4 * MAX_HEAVY, st));
        hc.hs = &hs;
        hc.out = HeavyOut{hrow, reinterpret_cast<unsigned long long*>(ws + L.heavy_items), out_b, out_p, capacity};
    }
    if ((s = partition_column<K>(static_cast<const K*>(d->build_keys), d->n_build, p, L, 0, ws,
                                 reinterpret_cast<uint32_t*>(ws + L.b_tuples), L.b_cap, E, PJ_STAGE_BUILD_HIST,
                                 st)) != PJ_OK)
        return s;
    if (hc.hs) {  // build rows of the heavy keys (timed with the build scatter)
        heavy_rows_kernel<K><<<static_cast<unsigned>(sm_count()) * 4, 512, 0, st>>>(static_cast<const K*>(d->build_keys),
                                                                        d->n_build, hs,
                                                                        const_cast<int32_t*>(hc.out.heavy_row));
        PJ_CUDA(cudaGetLastError());
    }
    const bool two = p->passes == 2;
    E.mark(PJ_STAGE_BUILD_PASS2, st);
    if (two && (s = partition_pass2<K>(p, L, 0, ws, reinterpret_cast<uint32_t*>(ws + L.b_tuples2), L.b_cap2, st)) !=
                   PJ_OK)
        return s;
    if ((s = partition_column<K>(static_cast<const K*>(d->probe_keys), d->n_probe, p, L, 1, ws,
                                 reinterpret_cast<uint32_t*>(ws + L.p_tuples), L.p_cap, E, PJ_STAGE_PROBE_HIST,
                                 st, hc)) != PJ_OK)
        return s;
    E.mark(PJ_STAGE_PROBE_PASS2, st);
    if (two && (s = partition_pass2<K>(p, L, 1, ws, reinterpret_cast<uint32_t*>(ws + L.p_tuples2), L.p_cap2, st)) !=
                   PJ_OK)
        return s;
    // the partitions the join reads: second-pass output for two-pass plans
    const size_t jb_off = two ? L.b_off2 : L.b_off, jp_off = two ? L.p_off2 : L.p_off;
    const int jb_items = two ? L.C : L.b_items, jp_items = two ? L.C : L.p_items;
    E.mark(PJ_STAGE_JOIN_PLAN, st);
    if (hc.hs) {  // the heavy pairs [0, H) precede every join chunk
        heavy_total_kernel<<<1, 32, 0, st>>>(hc.out.item_count, L.p_items, heavy_total,
                                             reinterpret_cast<unsigned long long*>(count));
        PJ_CUDA(cudaGetLastError());
    }

    const int cap_tuples = table_tuples(p);
    const bool hash_split = p->split_mode == PJ_SPLIT_HASH;
    const int position_chunk = std::max(16, cap_tuples / 16 * 16);
    join_items_kernel<<<(L.P + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<int64_t*>(ws + jb_off), reinterpret_cast<int64_t*>(ws + jp_off), jb_items, jp_items,
        L.P, reinterpret_cast<int32_t*>(ws + L.b_tot), reinterpret_cast<int32_t*>(ws + L.p_tot),
        hash_split ? cap_tuples : position_chunk, p->probe_chunk, hash_split ? 1 : 0, MAX_SPLIT_LOG2,
        reinterpret_cast<int32_t*>(ws + L.split), reinterpret_cast<int64_t*>(ws + L.items), status, nullptr);
    PJ_CUDA(cudaGetLastError());
    if ((s = launch_scan<int64_t>(reinterpret_cast<int64_t*>(ws + L.items), L.P, 1u,
                                  reinterpret_cast<int64_t*>(ws + L.item_off), reinterpret_cast<uint64_t*>(ws + L.i_tiles),
                                  ctr + CTR_ITILE, status, st)) != PJ_OK)
        return s;
    items_expand_kernel<<<L.P, 256, 0, st>>>(reinterpret_cast<int64_t*>(ws + L.item_off), L.P,
                                             reinterpret_cast<int32_t*>(ws + L.item_part), L.max_items, status);
    PJ_CUDA(cudaGetLastError());

    JoinArgs a{};
    a.build_tuples = reinterpret_cast<const uint32_t*>(ws + (two ? L.b_tuples2 : L.b_tuples));
    a.probe_tuples = reinterpret_cast<const uint32_t*>(ws + (two ? L.p_tuples2 : L.p_tuples));
    a.build_off = reinterpret_cast<const int64_t*>(ws + jb_off);
    a.probe_off = reinterpret_cast<const int64_t*>(ws + jp_off);
    a.b_items = jb_items;
    a.p_items = jp_items;
    a.P = L.P;
    // top hash bits the partition digits consumed
    a.digit_bits = (p->digit_mode == PJ_DIGIT_HASH ? p->bits1 : 0) + (two ? p->bits2 : 0);
    a.split = reinterpret_cast<const int32_t*>(ws + L.split);
    a.item_off = reinterpret_cast<const int64_t*>(ws + L.item_off);
    a.item_part = reinterpret_cast<const int32_t*>(ws + L.item_part);
    a.max_items = L.max_items;
    a.queue = ctr + CTR_QUEUE;
    a.cap = p->table_capacity;
    a.nb_log2 = table_nb_log2(d->n_build, p);
    a.row_bits = exact_row_bits(d->n_build);
    a.probe_chunk = p->probe_chunk;
    a.position_chunk = position_chunk;
    a.out_build = out_b;
    a.out_probe = out_p;
    a.capacity = capacity;
    a.count = reinterpret_cast<unsigned long long*>(count);
    a.status = status;
    a.cta_q = reinterpret_cast<int64_t*>(ws + L.cta_q);
    a.cta_last = reinterpret_cast<int64_t*>(ws + L.cta_last);
    a.seg = reinterpret_cast<int64_t*>(ws + L.seg);
    a.over_build = reinterpret_cast<int32_t*>(ws + L.over_b);
    a.over_probe = reinterpret_cast<int32_t*>(ws + L.over_p);
    a.over_cap = L.over_cap;
    a.max_ctas = L.max_ctas;
    a.base_count = heavy_total;
    E.mark(PJ_STAGE_JOIN, st);
    s = launch_join<K>(a, p->table_mode, d->unique_build_keys != 0, hash_split, p->slot_mode == PJ_SLOT_REF, st);
    if (s == PJ_OK && out_b && (pay_b || pay_p) && d->payload_bytes > 0) {
        const unsigned grid = static_cast<unsigned>(sm_count()) * 8;
        const auto* cnt = reinterpret_cast<const unsigned long long*>(count);
        if (d->payload_bytes == 4)
            gather_payload_kernel<int32_t><<<grid, 256, 0, st>>>(
                out_b, out_p, static_cast<const int32_t*>(d->build_payload), static_cast<const int32_t*>(d->probe_payload),
                static_cast<int32_t*>(pay_b), static_cast<int32_t*>(pay_p), cnt, capacity);
        else
            gather_payload_kernel<int64_t><<<grid, 256, 0, st>>>(
                out_b, out_p, static_cast<const int64_t*>(d->build_payload), static_cast<const int64_t*>(d->probe_payload),
                static_cast<int64_t*>(pay_b), static_cast<int64_t*>(pay_p), cnt, capacity);
        PJ_CUDA(cudaGetLastError());
    }
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

pj_status check_ws(const pj_join_desc* d, const pj_plan* p, void* ws, size_t ws_bytes, Layout* L)
{
    *L = make_layout(d, p);
    if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u) || ws_bytes < L->total) return PJ_ERR_WORKSPACE;
    return PJ_OK;
}

pj_status check_inputs(const pj_join_desc* d)
{
    if (d->n_build > 0 && !aligned16(d->build_keys)) return PJ_ERR_ALIGNMENT;
    if (d->n_probe > 0 && !aligned16(d->probe_keys)) return PJ_ERR_ALIGNMENT;
    return PJ_OK;
}

pj_status check_output(const pj_join_desc* d, const pj_output* out)
{
    if (!out || !out->count || out->capacity < 0) return PJ_ERR_INVALID;
    if (out->capacity > 0 && (!out->build_row || !out->probe_row)) return PJ_ERR_INVALID;
    // a payload output needs its payload column
    if (d && d->payload_bytes > 0) {
        if (out->build_payload_out && d->n_build > 0 && !d->build_payload) return PJ_ERR_INVALID;
        if (out->probe_payload_out && d->n_probe > 0 && !d->probe_payload) return PJ_ERR_INVALID;
    }
    return PJ_OK;
}

pj_status prepare(const pj_join_desc* d, const pj_plan* plan, void* ws, size_t ws_bytes, pj_plan* p, Layout* L)
{
    if (!valid_desc(d)) return PJ_ERR_INVALID;
    pj_status s = resolve_plan(d, plan, p);
    if (s != PJ_OK) return s;
    if ((s = check_inputs(d)) != PJ_OK) return s;
    return check_ws(d, p, ws, ws_bytes, L);
}

pj_status dispatch_join(const pj_join_desc* d, const pj_plan* p, const Layout& L, void* ws, const pj_output* out,
                        int64_t* count, cudaStream_t st, const StageEvents& E)
{
    uint8_t* w = static_cast<uint8_t*>(ws);
    int32_t* ob = out ? out->build_row : nullptr;
    int32_t* op = out ? out->probe_row : nullptr;
    const int64_t cap = out ? out->capacity : 0;
    void* pb = out ? out->build_payload_out : nullptr;
    void* pp = out ? out->probe_payload_out : nullptr;
    if (d->key_bytes == 4) return run_join<int32_t>(d, p, L, w, ob, op, cap, count, pb, pp, st, E);
    return run_join<int64_t>(d, p, L, w, ob, op, cap, count, pb, pp, st, E);
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

const char* pj_version(void) { return "partitioned_join_b200 0.2 (sm_100a)"; }

pj_status pj_plan_default(const pj_join_desc* d, pj_plan* p)
{
    if (!valid_desc(d) || !p) return PJ_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->passes = 1;
    p->digit_mode = PJ_DIGIT_HASH;
    p->table_mode = PJ_TABLE_BUCKET;
    p->slot_mode = PJ_SLOT_FAST;
    p->split_mode = d->unique_build_keys ? PJ_SPLIT_HASH : PJ_SPLIT_POSITION;
    p->max_fill = 0.5f;  // HASH_TABLE_OCC, hash_join_kernels.cuh:21
    p->table_capacity = max_table_capacity(d->key_bytes, p->table_mode);
    // Probe tuples per work item: at least 64 K, and large enough that a
    // partition of average size is one item (every extra item of a partition
    // rebuilds its table) -- about 8 items per SM over the whole join.  Only
    // partitions far above average (skewed probe keys) are split.
    {
        const int64_t per = (d->n_probe + static_cast<int64_t>(sm_count()) * 8 - 1) / (static_cast<int64_t>(sm_count()) * 8);
        p->probe_chunk = static_cast<int32_t>(std::min<int64_t>(std::max<int64_t>(1 << 16, (per + 15) / 16 * 16), 1 << 30));
    }
    p->scatter_ctas_per_sm = 1;
    p->hist_split = 2;
    auto pick_w = [&](int b) { return pick_wc(d->key_bytes, b); };
    auto bits_for = [&](int64_t cap) { return bits_for_table(d->n_build, cap); };
    int bits = bits_for(p->table_capacity);
    if (pick_w(bits) == 0) {
        // beyond one pass's fan-out: 4-byte COMPACT entries hold twice the
        // tuples per table, so large partitions need no split
        const int ccap = max_table_capacity(d->key_bytes, PJ_TABLE_COMPACT);
        // (only where partitions stay within an entry's 16-bit index)
        if (ccap > p->table_capacity && pick_w(bits_for(ccap)) != 0) {
            p->table_mode = PJ_TABLE_COMPACT;
            p->table_capacity = ccap;
            // the widest fan-out one pass makes: smaller build ranges keep
            // the fingerprint checks' loads in L2 (2^26 x 2^28 int64: 2048
            // partitions 7.2 ms, 4096 partitions 4.6 ms)
            bits = bits_for(ccap);
            while (bits < 16 && pick_w(bits + 1) != 0) ++bits;
        }
    }
    if (pick_w(bits) == 0 && p->table_mode == PJ_TABLE_BUCKET) {
        // beyond what one pass makes even for COMPACT tables: two passes
        // (the reference's radix plan, main.cu:240-248), BUCKET tables
        const int b1 = (bits + 1) / 2, b2 = bits - b1;
        const int w = pick_w(b1);
        if (b2 >= 1 && w != 0) {
            p->passes = 2;
            p->bits1 = b1;
            p->bits2 = b2;
            p->wc_tuples = w;
            return PJ_OK;
        }
    }
    while (bits > 0 && pick_w(bits) == 0) --bits;  // still beyond: hash splits absorb the rest
    p->bits1 = bits;
    p->wc_tuples = pick_w(bits);
    if (p->wc_tuples == 0) p->wc_tuples = d->key_bytes == 4 ? 4 : 8;
    if (p->table_mode == PJ_TABLE_COMPACT) {
        // EXACT tables (no build-tuple loads) where the expected largest
        // hashed partition (mean + 4 standard deviations) fits one
        const double m = static_cast<double>(d->n_build) / static_cast<double>(int64_t(1) << bits);
        const int cap_e = exact_table_capacity(d->key_bytes, exact_row_bits(d->n_build) - bits);
        if (cap_e > 0 && m + 4.0 * std::sqrt(m) + 1.0 <= cap_e) {
            p->table_mode = PJ_TABLE_EXACT;
            p->table_capacity = cap_e;
        }
    }
    return PJ_OK;
}

pj_status pj_plan_radix(const pj_join_desc* d, int32_t partitions_1, int32_t partitions_2, float factor, pj_plan* p)
{
    if (!valid_desc(d) || !p) return PJ_ERR_INVALID;
    auto pow2 = [](int32_t x) { return x > 0 && (x & (x - 1)) == 0; };
    if (!pow2(partitions_1) || (partitions_2 != 0 && !pow2(partitions_2))) return PJ_ERR_INVALID;  // main.cu:239-251
    if (!(factor > 0.0f)) return PJ_ERR_INVALID;
    pj_status s = pj_plan_default(d, p);
    if (s != PJ_OK) return s;
    const int b1 = ilog2_floor(partitions_1), b2 = partitions_2 ? ilog2_floor(partitions_2) : 0;
    p->passes = partitions_2 ? 2 : 1;
    p->bits1 = b1;
    p->bits2 = b2;
    p->digit_mode = PJ_DIGIT_RAW;  // the first pass's digit is raw key bits, as the reference's
    p->table_mode = PJ_TABLE_BUCKET;
    p->split_mode = PJ_SPLIT_POSITION;  // handle_skewed_data cuts partitions into build chunks by position
    p->wc_tuples = pick_wc(d->key_bytes, b1);
    if (p->wc_tuples == 0) return PJ_ERR_INVALID;  // beyond one scatter pass's fan-out
    // the build chunk ceil(factor * |R| / partitions) (partitioned_join.cuh:198-206), within one table
    const double parts = static_cast<double>(partitions_1) * (partitions_2 ? partitions_2 : 1);
    const double chunk = std::ceil(static_cast<double>(factor) * static_cast<double>(d->n_build) / parts);
    const int max_cap = max_table_capacity(d->key_bytes, PJ_TABLE_BUCKET);
    p->table_capacity = static_cast<int32_t>(std::min<double>(max_cap, std::max(64.0, chunk)));
    return check_plan(d, p);
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

pj_status pj_inner_join(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws, size_t ws_bytes,
                        pj_stream stream)
{
    pj_status s = check_output(d, out);
    if (s != PJ_OK) return s;
    pj_plan p;
    Layout L;
    if ((s = prepare(d, plan, ws, ws_bytes, &p, &L)) != PJ_OK) return s;
    return dispatch_join(d, &p, L, ws, out, out->count,
                         static_cast<cudaStream_t>(stream), StageEvents());
}

pj_status pj_inner_join_events(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws,
                               size_t ws_bytes, pj_stream stream, void* const* events)
{
    pj_status s = check_output(d, out);
    if (s != PJ_OK) return s;
    if (!events) return PJ_ERR_INVALID;
    for (int i = 0; i < PJ_NUM_STAGES; ++i)
        if (!events[i]) return PJ_ERR_INVALID;
    pj_plan p;
    Layout L;
    if ((s = prepare(d, plan, ws, ws_bytes, &p, &L)) != PJ_OK) return s;
    StageEvents E;
    E.ev = reinterpret_cast<cudaEvent_t*>(const_cast<void**>(events));
    return dispatch_join(d, &p, L, ws, out, out->count,
                         static_cast<cudaStream_t>(stream), E);
}

pj_status pj_inner_join_timed(const pj_join_desc* d, const pj_plan* plan, pj_output* out, void* ws,
                              size_t ws_bytes, pj_stream stream, float* stage_ms)
{
    pj_status s = check_output(d, out);
    if (s != PJ_OK) return s;
    if (!stage_ms) return PJ_ERR_INVALID;
    pj_plan p;
    Layout L;
    if ((s = prepare(d, plan, ws, ws_bytes, &p, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[PJ_NUM_STAGES];
    for (int i = 0; i < PJ_NUM_STAGES; ++i) PJ_CUDA(cudaEventCreate(&ev[i]));
    StageEvents E;
    E.ev = ev;
    s = dispatch_join(d, &p, L, ws, out, out->count, st, E);
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

pj_status pj_join_count(const pj_join_desc* d, const pj_plan* plan, int64_t* count_dev, void* ws, size_t ws_bytes,
                        pj_stream stream)
{
    if (!count_dev) return PJ_ERR_INVALID;
    pj_plan p;
    Layout L;
    pj_status s = prepare(d, plan, ws, ws_bytes, &p, &L);
    if (s != PJ_OK) return s;
    // no output columns: the join counts every match and writes none
    return dispatch_join(d, &p, L, ws, nullptr, count_dev, static_cast<cudaStream_t>(stream),
                         StageEvents());
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

pj_status pj_diag_scan_timeout(const pj_join_desc* d, const pj_plan* plan, void* ws, size_t ws_bytes,
                               int64_t withhold_tile, uint32_t spin_limit, pj_stream stream)
{
    pj_plan p;
    Layout L;
    pj_status s = prepare(d, plan, ws, ws_bytes, &p, &L);
    if (s != PJ_OK) return s;
    const int64_t m = static_cast<int64_t>(L.P1) * L.b_items;
    const int64_t ntiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    if (withhold_tile < 0 || withhold_tile + 1 >= ntiles || spin_limit == 0) return PJ_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    PJ_CUDA(cudaMemsetAsync(w, 0, L.ctrl_end, st));  // as a join starts: zero counts, tile states, status
    uint32_t* ctr = reinterpret_cast<uint32_t*>(w + L.counters);
    return launch_scan<uint32_t>(reinterpret_cast<const uint32_t*>(w + L.b_counts), m, 1u,
                                 reinterpret_cast<int64_t*>(w + L.b_off), reinterpret_cast<uint64_t*>(w + L.b_tiles),
                                 ctr + CTR_BTILE, reinterpret_cast<uint32_t*>(w + L.status), st,
                                 ScanWait{withhold_tile, spin_limit});
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
    if (!valid_wc(key_bytes, plan->wc_tuples)) return PJ_ERR_INVALID;
    pj_join_desc d{};
    d.build_keys = reinterpret_cast<const void*>(16);
    d.n_build = n;
    d.key_bytes = key_bytes;
    d.unique_build_keys = 1;
    const Layout L = make_layout(&d, plan);
    *tuples = plan->passes == 2 ? L.b_cap2 : L.b_cap;
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
    d.n_build = n;
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
    PJ_CUDA(cudaMemsetAsync(w, 0, L.ctrl_end, st));
    const bool two = plan->passes == 2;
    uint32_t* first = two ? reinterpret_cast<uint32_t*>(w + L.b_tuples) : static_cast<uint32_t*>(tuples);
    if (key_bytes == 4)
        s = partition_column<int32_t>(static_cast<const int32_t*>(keys), n, plan, L, 0, w, first, L.b_cap,
                                      StageEvents(), 0, st);
    else
        s = partition_column<int64_t>(static_cast<const int64_t*>(keys), n, plan, L, 0, w, first, L.b_cap,
                                      StageEvents(), 0, st);
    if (s != PJ_OK) return s;
    if (two) {
        s = key_bytes == 4 ? partition_pass2<int32_t>(plan, L, 0, w, static_cast<uint32_t*>(tuples), L.b_cap2, st)
                           : partition_pass2<int64_t>(plan, L, 0, w, static_cast<uint32_t*>(tuples), L.b_cap2, st);
        if (s != PJ_OK) return s;
    }
    partition_bounds_kernel<<<(L.P + 1 + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<int64_t*>(w + (two ? L.b_off2 : L.b_off)), two ? L.C : L.b_items, L.P, offsets);
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
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    const int P = 1 << p.bits1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Histograms of the build keys under both digit sources, in the
    // workspace's count area (P x items >= 2P words).
    int32_t* hist = reinterpret_cast<int32_t*>(static_cast<uint8_t*>(ws) + L.b_counts);
    if ((s = pj_radix_histogram(d->build_keys, d->n_build, d->key_bytes, PJ_DIGIT_RAW, p.bits1, 0, 0, hist, stream)) !=
        PJ_OK)
        return s;
    if ((s = pj_radix_histogram(d->build_keys, d->n_build, d->key_bytes, PJ_DIGIT_HASH, p.bits1, 0, 0, hist + P,
                                stream)) != PJ_OK)
        return s;
    // A sample of the probe keys for the heavy-key path (unique build keys:
    // a heavy probe key then has at most one build row).
    const bool sample = d->unique_build_keys && d->n_probe >= HEAVY_MIN_PROBE;
    std::vector<int64_t> keys_h(sample ? HEAVY_SAMPLES : 0);
    int64_t* sample_d = reinterpret_cast<int64_t*>(static_cast<uint8_t*>(ws) + L.sample);
    if (sample) {
        if (d->key_bytes == 4)
            sample_keys_kernel<int32_t><<<HEAVY_SAMPLES / 256, 256, 0, st>>>(
                static_cast<const int32_t*>(d->probe_keys), d->n_probe, HEAVY_SAMPLES, sample_d);
        else
            sample_keys_kernel<int64_t><<<HEAVY_SAMPLES / 256, 256, 0, st>>>(
                static_cast<const int64_t*>(d->probe_keys), d->n_probe, HEAVY_SAMPLES, sample_d);
        PJ_CUDA(cudaGetLastError());
    }
    std::vector<int32_t> host(2 * static_cast<size_t>(P));
    cudaError_t e = cudaMemcpyAsync(host.data(), hist, sizeof(int32_t) * 2 * P, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && sample)
        e = cudaMemcpyAsync(keys_h.data(), sample_d, sizeof(int64_t) * HEAVY_SAMPLES, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        last_cuda_error() = e;
        return PJ_ERR_CUDA;
    }
    if (sample) {
        // the path pays a lookup for every probe key: worth it only when the
        // heavy keys carry a large share of the probe side
        const double share = heavy_from_sample(keys_h, HEAVY_MIN_SAMPLES, &p);
        if (share < HEAVY_MIN_SHARE) p.n_heavy = 0;
    }
    int64_t raw_max = 0, hash_max = 0;
    for (int i = 0; i < P; ++i) {
        raw_max = std::max<int64_t>(raw_max, host[i]);
        hash_max = std::max<int64_t>(hash_max, host[P + i]);
    }
    // (an EXACT default is decided again below from the hashed partitions)
    if (p.table_mode == PJ_TABLE_EXACT) {
        p.table_mode = PJ_TABLE_COMPACT;
        p.table_capacity = max_table_capacity(d->key_bytes, PJ_TABLE_COMPACT);
    }
    // Raw key bits are free to compute: keep them (the reference's digits)
    // when their largest partition is no worse than the hashed one's.
    p.digit_mode = raw_max <= hash_max ? PJ_DIGIT_RAW : PJ_DIGIT_HASH;
    const int64_t mx = std::min(raw_max, hash_max);
    // a COMPACT entry addresses 65536 tuples of a build range (padding included)
    if (p.table_mode == PJ_TABLE_COMPACT &&
        mx + static_cast<int64_t>(L.b_items) * (p.wc_tuples - 1) > COMPACT_RANGE) {
        p.table_mode = PJ_TABLE_BUCKET;
        p.table_capacity = max_table_capacity(d->key_bytes, PJ_TABLE_BUCKET);
    }
    // EXACT tables instead of COMPACT ones (no build-tuple loads) where hash
    // digits keep the largest partition within one -- unless the heavy-key
    // path takes most probe rows: then the join has few lookups to save and
    // the hash digits' histogram costs more (2^26 x 2^28 int64 at Zipf 1.5:
    // 5.06 ms with EXACT tables, 4.84 ms without)
    int64_t mx_plan = mx;
    if (p.passes == 1 && p.table_mode == PJ_TABLE_COMPACT && p.n_heavy == 0) {
        const int cap_e = exact_table_capacity(d->key_bytes, exact_row_bits(d->n_build) - p.bits1);
        if (cap_e > 0 && hash_max <= cap_e) {
            p.table_mode = PJ_TABLE_EXACT;
            p.digit_mode = PJ_DIGIT_HASH;
            p.table_capacity = cap_e;
            mx_plan = hash_max;
        }
    }
    const int64_t cap = table_tuples(&p);
    // Hash splits cannot separate repeated keys: a partition beyond what
    // 2^MAX_SPLIT_LOG2 tables hold (duplicates) takes the position split.
    if (mx_plan > cap * (int64_t(1) << MAX_SPLIT_LOG2) / 2) p.split_mode = PJ_SPLIT_POSITION;
    *plan = p;
    return PJ_OK;
}

// ---- learned planner ------------------------------------------------------

pj_status pj_plan_features(const pj_join_desc* d, void* ws, size_t ws_bytes, float* features, pj_plan* heavy,
                           pj_stream stream)
{
    if (!valid_desc(d) || !features) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = pj_plan_default(d, &p);
    if (s != PJ_OK) return s;
    Layout L;
    if ((s = check_ws(d, &p, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint8_t* w = static_cast<uint8_t*>(ws);
    float* feat_d = reinterpret_cast<float*>(w + L.learn);
    int64_t* sample_d = reinterpret_cast<int64_t*>(w + L.sample);
    const int samples = d->n_probe > 0 ? static_cast<int>(std::min<int64_t>(std::max<int64_t>(d->n_probe / 100, 4096),
                                                                            HEAVY_SAMPLES))
                                       : 0;
    const float lnb = static_cast<float>(std::log2(static_cast<double>(std::max<int64_t>(d->n_build, 1))));
    const float lnp = static_cast<float>(std::log2(static_cast<double>(std::max<int64_t>(d->n_probe, 1))));
    if (samples > 0 && !aligned16(d->probe_keys)) return PJ_ERR_ALIGNMENT;
    if (d->key_bytes == 4)
        plan_features_kernel<int32_t><<<1, SKETCH_BINS, 0, st>>>(static_cast<const int32_t*>(d->probe_keys), d->n_probe,
                                                                 samples, sample_d, feat_d, lnb, lnp, 4.0f,
                                                                 d->unique_build_keys ? 1.0f : 0.0f);
    else
        plan_features_kernel<int64_t><<<1, SKETCH_BINS, 0, st>>>(static_cast<const int64_t*>(d->probe_keys), d->n_probe,
                                                                 samples, sample_d, feat_d, lnb, lnp, 8.0f,
                                                                 d->unique_build_keys ? 1.0f : 0.0f);
    PJ_CUDA(cudaGetLastError());
    std::vector<int64_t> keys_h(static_cast<size_t>(heavy ? samples : 0));
    PJ_CUDA(cudaMemcpyAsync(features, feat_d, sizeof(float) * PJ_MLP_FEATURES, cudaMemcpyDeviceToHost, st));
    if (heavy && samples > 0)
        PJ_CUDA(cudaMemcpyAsync(keys_h.data(), sample_d, sizeof(int64_t) * samples, cudaMemcpyDeviceToHost, st));
    PJ_CUDA(cudaStreamSynchronize(st));
    if (heavy) {
        std::memset(heavy, 0, sizeof(*heavy));
        if (d->unique_build_keys && samples > 0)
            heavy_from_sample(keys_h, std::max(2, samples / 2048), heavy);
    }
    return PJ_OK;
}

pj_status pj_plan_candidate(const pj_join_desc* d, int32_t candidate, const pj_plan* heavy, pj_plan* plan)
{
    if (!valid_desc(d) || !plan || candidate < 0 || candidate >= PJ_PLAN_CANDIDATES) return PJ_ERR_INVALID;
    pj_plan p;
    pj_status s = pj_plan_default(d, &p);
    if (s != PJ_OK) return s;
    p.n_heavy = 0;
    int max_bits = 0;
    for (int b = 0; b <= 16; ++b)
        if (pick_wc(d->key_bytes, b) != 0) max_bits = b;
    const double n = static_cast<double>(std::max<int64_t>(d->n_build, 1));
    auto largest = [&](int bits) {  // expected largest hashed partition: mean + 4 standard deviations
        const double m = n / static_cast<double>(int64_t(1) << bits);
        return m + 4.0 * std::sqrt(m) + 1.0;
    };
    if (candidate < 27) {
        // table layout x radix bits (-1, 0, +1 around the layout's own width) x heavy-key set
        const int table = candidate / 9, delta = (candidate % 9) / 3 - 1, heavy_mode = candidate % 3;
        p.digit_mode = PJ_DIGIT_HASH;
        p.split_mode = d->unique_build_keys ? PJ_SPLIT_HASH : PJ_SPLIT_POSITION;
        if (table == 0 || table == 1) {
            p.table_mode = table == 0 ? PJ_TABLE_BUCKET : PJ_TABLE_COMPACT;
            p.table_capacity = max_table_capacity(d->key_bytes, p.table_mode);
            // (a COMPACT choice whose partitions exceed an entry's 65536-tuple
            // index range is valid here and overflows on the device: the
            // caller then falls back to the exact plan)
            p.bits1 = std::min(std::max(bits_for_table(d->n_build, p.table_capacity) + delta, 0), max_bits);
        } else {
            // EXACT: hash digits and enough buckets that an entry fixes the key
            const int ccap = max_table_capacity(d->key_bytes, PJ_TABLE_COMPACT);
            p.bits1 = std::min(std::max(bits_for_table(d->n_build, ccap) + delta, 0), max_bits);
            const int cap_e = exact_table_capacity(d->key_bytes, exact_row_bits(d->n_build) - p.bits1);
            if (cap_e == 0 || largest(p.bits1) > cap_e) return PJ_ERR_INVALID;
            p.table_mode = PJ_TABLE_EXACT;
            p.table_capacity = cap_e;
            if (!d->unique_build_keys) return PJ_ERR_INVALID;
        }
        p.wc_tuples = pick_wc(d->key_bytes, p.bits1);
        if (p.wc_tuples == 0) return PJ_ERR_INVALID;
        if (heavy_mode != 0) {
            // the sample's heavy keys (most frequent first): all of them, or the 16 most frequent
            if (!heavy || !d->unique_build_keys || heavy->n_heavy <= 0) return PJ_ERR_INVALID;
            p.n_heavy = std::min(heavy_mode == 1 ? heavy->n_heavy : std::min(heavy->n_heavy, 16), PJ_MAX_HEAVY);
            for (int i = 0; i < p.n_heavy; ++i) p.heavy_keys[i] = heavy->heavy_keys[i];
            if (p.table_mode == PJ_TABLE_EXACT) return PJ_ERR_INVALID;  // the heavy path keeps COMPACT/BUCKET tables
        }
    } else if (candidate == PJ_PLAN_CANDIDATE_EXACT) {
        return PJ_ERR_INVALID;  // pj_plan_exact's plan: made on the device by pj_plan_learned
    } else {
        // two radix passes, BUCKET tables: the BUCKET width + 0 or 1 bit, split evenly
        p.table_mode = PJ_TABLE_BUCKET;
        p.digit_mode = PJ_DIGIT_HASH;
        p.table_capacity = max_table_capacity(d->key_bytes, PJ_TABLE_BUCKET);
        const int bits = bits_for_table(d->n_build, p.table_capacity) + (candidate - 27);
        if (bits < 2) return PJ_ERR_INVALID;
        p.passes = 2;
        p.bits1 = (bits + 1) / 2;
        p.bits2 = bits - p.bits1;
        p.wc_tuples = pick_wc(d->key_bytes, p.bits1);
        if (p.wc_tuples == 0 || pass2_wc(d->key_bytes, &p) == 0) return PJ_ERR_INVALID;
        p.split_mode = d->unique_build_keys ? PJ_SPLIT_HASH : PJ_SPLIT_POSITION;
    }
    if ((s = check_plan(d, &p)) != PJ_OK) return s;
    *plan = p;
    return PJ_OK;
}

pj_status pj_plan_learned(const pj_join_desc* d, const float* params, void* ws, size_t ws_bytes, pj_plan* plan,
                          float* scores, pj_stream stream)
{
    if (!valid_desc(d) || !plan || !params) return PJ_ERR_INVALID;
    float feat[PJ_MLP_FEATURES];
    pj_plan heavy;
    pj_status s = pj_plan_features(d, ws, ws_bytes, feat, &heavy, stream);
    if (s != PJ_OK) return s;
    pj_plan p0;
    pj_plan_default(d, &p0);
    Layout L;
    if ((s = check_ws(d, &p0, ws, ws_bytes, &L)) != PJ_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* feat_d = reinterpret_cast<float*>(static_cast<uint8_t*>(ws) + L.learn);
    const pj_mlp_dims dims{PJ_MLP_FEATURES, PJ_MLP_HIDDEN, PJ_MLP_HIDDEN, PJ_PLAN_CANDIDATES};
    float* acts_d = feat_d + PJ_MLP_FEATURES;
    float* out_d = acts_d + 4 * PJ_MLP_HIDDEN;
    static_assert((PJ_MLP_FEATURES + 4 * PJ_MLP_HIDDEN + PJ_PLAN_CANDIDATES) * sizeof(float) <= LEARN_BYTES,
                  "learned-planner scratch");
    if ((s = pj_mlp_forward(params, &dims, feat_d, 1, acts_d, out_d, stream)) != PJ_OK) return s;
    float out[PJ_PLAN_CANDIDATES];
    PJ_CUDA(cudaMemcpyAsync(out, out_d, sizeof(out), cudaMemcpyDeviceToHost, st));
    PJ_CUDA(cudaStreamSynchronize(st));
    if (scores) std::memcpy(scores, out, sizeof(out));
    int order[PJ_PLAN_CANDIDATES];
    for (int i = 0; i < PJ_PLAN_CANDIDATES; ++i) order[i] = i;
    std::sort(order, order + PJ_PLAN_CANDIDATES, [&](int a, int b) { return out[a] < out[b]; });
    for (int c : order) {
        if (c == PJ_PLAN_CANDIDATE_EXACT) return pj_plan_exact(d, ws, ws_bytes, plan, stream);
        if (pj_plan_candidate(d, c, &heavy, plan) == PJ_OK) return PJ_OK;
    }
    return pj_plan_default(d, plan);
}

}  // extern "C"

// ===========================================================================
// The partitioned joins of a batch, run together (pj_internal.h).
namespace pj_internal {

namespace {

constexpr int64_t SEG_CHUNK = 1 << 16;  // rows of one scatter item of a batch segment

template <typename K>
pj_status large_batch_run_t(const LargeBatch& lb, void* ws, uint32_t* status, cudaStream_t st)
{
    uint8_t* w = static_cast<uint8_t*>(ws);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(w + lb.o_counters);
    uint32_t* counts = reinterpret_cast<uint32_t*>(w + lb.o_counts);
    int32_t* totals = reinterpret_cast<int32_t*>(w + lb.o_totals);
    int64_t* off = reinterpret_cast<int64_t*>(w + lb.o_off);
    uint32_t* tuples = reinterpret_cast<uint32_t*>(w + lb.o_tuples);
    const SegItem* items = reinterpret_cast<const SegItem*>(w + lb.o_items);
    const int n_items = static_cast<int>(lb.seg.size());
    PJ_CUDA(cudaMemsetAsync(w + lb.o_ctrl, 0, lb.ctrl_bytes, st));
    const int n_jobs = static_cast<int>(lb.joins.size());
    zero_job_counts_kernel<<<(n_jobs + 255) / 256, 256, 0, st>>>(reinterpret_cast<const JobOut*>(w + lb.o_outs), n_jobs);
    PJ_CUDA(cudaGetLastError());
    // histogram, scan, scatter over every segment of every join
    const size_t hsmem = 4 * static_cast<size_t>((lb.Pmax + 3) & ~3);
    PJ_CUDA(set_smem(hist_seg_kernel<K>, hsmem));
    hist_seg_kernel<K><<<static_cast<unsigned>(n_items) * 2, HIST_THREADS, hsmem, st>>>(items, 2, counts, totals);
    PJ_CUDA(cudaGetLastError());
    pj_status s;
    if ((s = launch_scan<uint32_t>(counts, lb.n_counts, static_cast<uint32_t>(lb.W), off,
                                   reinterpret_cast<uint64_t*>(w + lb.o_tiles), ctr + CTR_BTILE, status, st)) != PJ_OK)
        return s;
    constexpr int VT = sizeof(K) == 4 ? 4 : 2;
    const size_t ssmem = scatter_smem(sizeof(K), lb.wc_cap, lb.Pmax);
    const uint32_t out_cap = static_cast<uint32_t>(std::min<int64_t>(lb.tuples, UINT32_MAX));
    const int sgrid = std::min(n_items, sm_count());
    switch (lb.W) {
    case 4: {
        auto* k = scatter_seg_kernel<K, SC_THREADS, VT, 4>;
        PJ_CUDA(set_smem(k, ssmem));
        k<<<sgrid, SC_THREADS, ssmem, st>>>(items, n_items, lb.Pmax, lb.wc_cap, off, tuples, out_cap, status);
        break;
    }
    case 2: {
        auto* k = scatter_seg_kernel<K, SC_THREADS, VT, 2>;
        PJ_CUDA(set_smem(k, ssmem));
        k<<<sgrid, SC_THREADS, ssmem, st>>>(items, n_items, lb.Pmax, lb.wc_cap, off, tuples, out_cap, status);
        break;
    }
    default: return PJ_ERR_INVALID;
    }
    PJ_CUDA(cudaGetLastError());
    // work split over all partitions, then one join launch
    const PartRef* parts = reinterpret_cast<const PartRef*>(w + lb.o_parts);
    const int cap_tuples = lb.table_cap;
    const bool hash_split = lb.unique;
    const int position_chunk = std::max(16, cap_tuples / 16 * 16);
    join_items_kernel<<<(lb.G + 255) / 256, 256, 0, st>>>(
        off, off, 1, 1, lb.G, totals, totals + lb.G, hash_split ? cap_tuples : position_chunk, lb.probe_chunk,
        hash_split ? 1 : 0, MAX_SPLIT_LOG2, reinterpret_cast<int32_t*>(w + lb.o_split),
        reinterpret_cast<int64_t*>(w + lb.o_jitems), status, parts);
    PJ_CUDA(cudaGetLastError());
    if ((s = launch_scan<int64_t>(reinterpret_cast<int64_t*>(w + lb.o_jitems), lb.G, 1u,
                                  reinterpret_cast<int64_t*>(w + lb.o_item_off),
                                  reinterpret_cast<uint64_t*>(w + lb.o_itiles), ctr + CTR_ITILE, status, st)) != PJ_OK)
        return s;
    items_expand_kernel<<<lb.G, 256, 0, st>>>(reinterpret_cast<int64_t*>(w + lb.o_item_off), lb.G,
                                              reinterpret_cast<int32_t*>(w + lb.o_item_part), lb.max_items, status);
    PJ_CUDA(cudaGetLastError());
    JoinArgs a{};
    a.build_tuples = a.probe_tuples = tuples;
    a.build_off = a.probe_off = off;
    a.b_items = a.p_items = 1;
    a.P = lb.G;
    a.split = reinterpret_cast<const int32_t*>(w + lb.o_split);
    a.item_off = reinterpret_cast<const int64_t*>(w + lb.o_item_off);
    a.item_part = reinterpret_cast<const int32_t*>(w + lb.o_item_part);
    a.max_items = lb.max_items;
    a.queue = ctr + CTR_QUEUE;
    a.cap = lb.table_cap;
    a.nb_log2 = lb.nb_log2;
    a.probe_chunk = lb.probe_chunk;
    a.position_chunk = position_chunk;
    a.status = status;
    a.parts = parts;
    a.outs = reinterpret_cast<const JobOut*>(w + lb.o_outs);
    auto launch = [&](auto* kern) -> pj_status {
        const size_t smem = JoinSmem<K, TABLE_BUCKET>::bytes(a.cap, a.nb_log2);
        PJ_CUDA(set_smem(kern, smem));
        int per_sm = 0;
        PJ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, JN_THREADS, smem));
        per_sm = std::min(std::max(per_sm, 1), MAX_JOIN_CTAS_PER_SM);
        kern<<<sm_count() * per_sm, JN_THREADS, smem, st>>>(a);
        PJ_CUDA(cudaGetLastError());
        return PJ_OK;
    };
    if (lb.unique) return launch(join_kernel<K, TABLE_BUCKET, true, true, false, JN_THREADS, true>);
    return launch(join_kernel<K, TABLE_BUCKET, false, false, false, JN_THREADS, true>);
}

}  // namespace

pj_status large_batch_layout(const pj_join_desc* descs, const std::vector<int>& joins, int bits_delta, LargeBatch* out)
{
    LargeBatch lb;
    if (joins.empty()) {
        *out = lb;
        return PJ_OK;
    }
    lb.key_bytes = descs[joins[0]].key_bytes;
    lb.table_cap = max_table_capacity(lb.key_bytes, PJ_TABLE_BUCKET);
    lb.nb_log2 = bucket_nb_log2(lb.table_cap);
    int64_t probe_total = 0;
    struct J { int idx, bits; };
    std::vector<J> take;
    for (int i : joins) {
        const pj_join_desc& d = descs[i];
        if (!valid_desc(&d) || d.key_bytes != lb.key_bytes) return PJ_ERR_INVALID;
        if (d.n_build == 0 || d.n_probe == 0) continue;  // nothing to join: the count stays 0
        const int bits = std::max(0, bits_for_table(d.n_build, lb.table_cap) + bits_delta);
        if (bits > LARGE_BATCH_MAX_BITS) continue;  // run alone (the segment kernels load keys one by one: any alignment)
        take.push_back({i, bits});
        lb.unique = lb.unique && d.unique_build_keys != 0;
        probe_total += d.n_probe;
    }
    for (const J& j : take) lb.Pmax = std::max(lb.Pmax, 1 << j.bits);
    lb.W = pick_wc(lb.key_bytes, ilog2_floor(lb.Pmax));
    if (lb.W == 0) return PJ_ERR_INVALID;
    lb.wc_cap = wc_cap(lb.key_bytes, lb.W, lb.Pmax, SC_THREADS * (lb.key_bytes == 4 ? 4 : 2), 0);
    // probe chunks: about 8 work items per SM over the whole batch
    {
        const int64_t per = (probe_total + static_cast<int64_t>(sm_count()) * 8 - 1) / (static_cast<int64_t>(sm_count()) * 8);
        lb.probe_chunk = static_cast<int32_t>(std::min<int64_t>(std::max<int64_t>(1 << 14, (per + 15) / 16 * 16), 1 << 30));
    }
    // partitions over all joins: build totals go to [0, G), probe totals to [G, 2G)
    lb.G = 0;
    for (const J& j : take) lb.G += 1 << j.bits;
    int64_t cnt = 0, tup = 0, max_items = 0;
    int g = 0;
    for (const J& j : take) {
        const pj_join_desc& d = descs[j.idx];
        const int P = 1 << j.bits;
        DigitFn f{PJ_DIGIT_HASH, j.bits ? 32 - j.bits : 0, static_cast<uint32_t>(P - 1)};
        int64_t base[2];
        int32_t nit[2];
        for (int side = 0; side < 2; ++side) {
            const int64_t n = side == 0 ? d.n_build : d.n_probe;
            const int items = static_cast<int>(std::max<int64_t>(1, (n + SEG_CHUNK - 1) / SEG_CHUNK));
            const int64_t chunk = chunk_for(n, items);
            base[side] = cnt;
            nit[side] = items;
            for (int i = 0; i < items; ++i) {
                SegItem it{};
                it.keys = side == 0 ? d.build_keys : d.probe_keys;
                it.lo = std::min<int64_t>(n, static_cast<int64_t>(i) * chunk);
                it.hi = std::min<int64_t>(n, it.lo + chunk);
                it.cnt_base = cnt;
                it.seg_items = items;
                it.item = i;
                it.tot_base = side == 0 ? g : lb.G + g;
                it.P = P;
                it.f = f;
                lb.seg.push_back(it);
            }
            cnt += static_cast<int64_t>(P) * items;
            tup += part_capacity(n, P, items, lb.W);
        }
        for (int p = 0; p < P; ++p) {
            PartRef r{};
            r.b_at = base[0] + static_cast<int64_t>(p) * nit[0];
            r.p_at = base[1] + static_cast<int64_t>(p) * nit[1];
            r.b_items = nit[0];
            r.p_items = nit[1];
            r.job = static_cast<int32_t>(lb.joins.size());
            r.digit_bits = j.bits;
            lb.parts.push_back(r);
        }
        // work items: each partition's build pieces (hash pieces, or
        // table-sized position pieces) times its probe chunks, as make_layout
        const int64_t per_piece = std::max<int64_t>(16, lb.table_cap / 16 * 16);
        const int64_t max_pieces = std::max<int64_t>(static_cast<int64_t>(P) << MAX_SPLIT_LOG2,
                                                     P + part_capacity(d.n_build, P, nit[0], lb.W) / per_piece);
        const int64_t max_chunks = P + part_capacity(d.n_probe, P, nit[1], lb.W) / lb.probe_chunk + 1;
        max_items += std::min<int64_t>(max_pieces * max_chunks, static_cast<int64_t>(P) * 4096 + max_pieces + max_chunks);
        lb.joins.push_back(j.idx);
        g += P;
    }
    lb.n_counts = cnt;
    lb.tuples = tup + 64;
    if (lb.tuples >= static_cast<int64_t>(UINT32_MAX)) return PJ_ERR_INVALID;
    lb.max_items = std::min<int64_t>(max_items, int64_t(1) << 30);
    lb.tiles_n = (lb.n_counts + SCAN_TILE - 1) / SCAN_TILE + 1;
    lb.itiles_n = (lb.G + SCAN_TILE - 1) / SCAN_TILE + 1;
    size_t o = 0;
    auto take_b = [&](size_t bytes) { const size_t at = o; o = align_up(o + bytes, 256); return at; };
    lb.o_ctrl = take_b(0);
    lb.o_counters = take_b(4 * 8);
    lb.o_counts = take_b(4 * static_cast<size_t>(lb.n_counts));
    lb.o_totals = take_b(4 * 2 * static_cast<size_t>(lb.G));
    lb.o_tiles = take_b(8 * static_cast<size_t>(lb.tiles_n));
    lb.o_itiles = take_b(8 * static_cast<size_t>(lb.itiles_n));
    lb.ctrl_bytes = o - lb.o_ctrl;
    lb.o_items = take_b(sizeof(SegItem) * lb.seg.size());
    lb.o_parts = take_b(sizeof(PartRef) * lb.parts.size());
    lb.o_outs = take_b(sizeof(JobOut) * lb.joins.size());
    lb.o_off = take_b(8 * static_cast<size_t>(lb.n_counts + 1));
    lb.o_split = take_b(4 * static_cast<size_t>(lb.G));
    lb.o_jitems = take_b(8 * static_cast<size_t>(lb.G));
    lb.o_item_off = take_b(8 * static_cast<size_t>(lb.G + 1));
    lb.o_item_part = take_b(4 * static_cast<size_t>(lb.max_items));
    lb.o_tuples = take_b(4 * static_cast<size_t>(tuple_words(lb.key_bytes)) * lb.tuples + 64);
    lb.total = o;
    *out = std::move(lb);
    return PJ_OK;
}

pj_status large_batch_upload(const LargeBatch& lb, const pj_output* outs, void* ws, cudaStream_t st)
{
    if (lb.joins.empty()) return PJ_OK;
    uint8_t* w = static_cast<uint8_t*>(ws);
    std::vector<JobOut> jo(lb.joins.size());
    for (size_t i = 0; i < lb.joins.size(); ++i) {
        const pj_output& o = outs[lb.joins[i]];
        jo[i] = JobOut{o.capacity > 0 ? o.build_row : nullptr, o.probe_row, o.capacity,
                       reinterpret_cast<unsigned long long*>(o.count)};
        if (o.capacity == 0) jo[i].out_build = nullptr;
    }
    PJ_CUDA(cudaMemcpyAsync(w + lb.o_items, lb.seg.data(), sizeof(SegItem) * lb.seg.size(), cudaMemcpyHostToDevice, st));
    PJ_CUDA(cudaMemcpyAsync(w + lb.o_parts, lb.parts.data(), sizeof(PartRef) * lb.parts.size(), cudaMemcpyHostToDevice,
                            st));
    PJ_CUDA(cudaMemcpyAsync(w + lb.o_outs, jo.data(), sizeof(JobOut) * jo.size(), cudaMemcpyHostToDevice, st));
    PJ_CUDA(cudaStreamSynchronize(st));
    return PJ_OK;
}

pj_status large_batch_run(const LargeBatch& lb, void* ws, uint32_t* status, cudaStream_t st)
{
    if (lb.joins.empty()) return PJ_OK;
    return lb.key_bytes == 4 ? large_batch_run_t<int32_t>(lb, ws, status, st)
                             : large_batch_run_t<int64_t>(lb, ws, status, st);
}

}  // namespace pj_internal
