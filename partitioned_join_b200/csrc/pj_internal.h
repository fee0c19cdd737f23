// pj_internal.h -- C++ interfaces shared by the library's own translation
// units (pj_api.cu, pj_batch.cu).  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pj.h"
#include "pj_types.cuh"

namespace pj_internal {

// The partitioned joins of a batch, run together: one histogram, one scan
// and one scatter launch over both key columns of every join, then one
// work-split and one join launch over all their partitions.  Each join has
// its own radix width (hash digits, BUCKET tables); matches go to the
// join's own output at exact positions.
struct LargeBatch {
    std::vector<int> joins;       // indices (into the batch) of the joins taken
    std::vector<pj::SegItem> seg; // scatter items of all segments (device copy at o_items)
    std::vector<pj::PartRef> parts;  // all partitions (device copy at o_parts)
    int key_bytes = 4;
    bool unique = true;           // every join has unique build keys
    int G = 0;                    // partitions over all joins
    int64_t n_counts = 0;         // counters over all segments
    int Pmax = 1, W = 4, wc_cap = 4;
    int64_t tuples = 0;           // tuple buffer capacity (tuples)
    int64_t max_items = 0;        // join work items the buffers hold
    int table_cap = 0, nb_log2 = 0, probe_chunk = 0;
    size_t o_ctrl = 0, ctrl_bytes = 0;  // zeroed by every run: status copy, counters, counts, totals, tiles
    size_t o_counters = 0, o_counts = 0, o_totals = 0, o_tiles = 0, o_itiles = 0;
    size_t o_items = 0, o_parts = 0, o_outs = 0, o_off = 0, o_split = 0, o_jitems = 0, o_item_off = 0,
           o_item_part = 0, o_tuples = 0;
    int64_t tiles_n = 0, itiles_n = 0;
    size_t total = 0;             // bytes
};

// Largest radix width (bits) of a join the batched path takes; wider joins
// run pj_inner_join on their own.
constexpr int LARGE_BATCH_MAX_BITS = 10;

// Plans the batched path for descs[joins] (bits_delta widens or narrows every
// join's radix width).  Sizes only: no device work.  Joins the path cannot
// take are left out of lb->joins.
pj_status large_batch_layout(const pj_join_desc* descs, const std::vector<int>& joins, int bits_delta,
                             LargeBatch* lb);

// Writes the item, partition and output tables into the region at ws
// (asynchronous on st; the host tables must outlive the copy, so callers
// synchronise before releasing lb).
pj_status large_batch_upload(const LargeBatch& lb, const pj_output* outs, void* ws, cudaStream_t st);

// Enqueues the batched path (kernels only: capturable in a CUDA graph).
// Device conditions are ORed into *status.
pj_status large_batch_run(const LargeBatch& lb, void* ws, uint32_t* status, cudaStream_t st);

}  // namespace pj_internal
