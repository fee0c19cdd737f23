// pj_types.cuh -- plain descriptors shared by the kernels and by the
// library's host code for batches of joins (no kernels: safe to include in
// every translation unit).
#pragma once

#include <cstdint>

#include "pj_device.cuh"

namespace pj {

// Scatter item of a batch of joins: one histogram and one scatter launch
// cover the key columns of many joins.  Each join side is a "segment" with its own
// partition count and digit; its columns are cut into items, and item i of a
// segment with P partitions and I items counts into
// counts[cnt_base + p * I + i].  One look-back scan over all segments' counts
// then lays every segment out in one shared tuple buffer: partition p of a
// segment is [off[cnt_base + p * I], off[cnt_base + (p + 1) * I]).  Rows stored
// in the tuples are rows of the segment's own column.
struct SegItem {
    const void* keys;  // the segment's key column
    int64_t lo, hi;    // this item's rows [lo, hi)
    int64_t cnt_base;  // first counter (and offset) of the segment
    int32_t seg_items; // items of the segment
    int32_t item;      // this item's index in the segment
    int32_t tot_base;  // first per-partition total of the segment
    int32_t P;         // partitions of the segment
    DigitFn f;         // the segment's digit (HASH digits)
};

// Partition of a batch of joins (pj_join_batch): the join kernel sees the
// partitions of many joins at once.  Partition g of the batch is partition p of one join side
// pair laid out by the segment scan: its build tuples are
// [build_off[b_at], build_off[b_at + b_items]), its probe tuples likewise,
// and its matches go to that join's output columns.
struct PartRef {
    int64_t b_at, p_at;      // offset index of the partition's first build / probe segment
    int32_t b_items, p_items;  // segments per partition on each side
    int32_t job;             // the join (index into JoinArgs::outs)
    int32_t digit_bits;      // top hash bits the join's digits consumed
};
struct JobOut {
    int32_t* out_build;           // nullptr: count only
    int32_t* out_probe;
    int64_t capacity;
    unsigned long long* count;    // device int64, zeroed before the launch
};

}  // namespace pj
