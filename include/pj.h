/*
 * pj.h -- C ABI of the B200-native radix-partitioned inner equi-join.
 *
 * Replaces the reference's `partitioned_join` stage sequence
 * (main.cu:762-892), whose stages are header templates called with raw
 * device pointers:
 *   partition_input_tables_pass_one   src/partitioned_join.cuh:51-107
 *   partition_input_tables_pass_two   src/partitioned_join.cuh:110-175
 *   combined_histogram_pass           src/partitioned_join.cuh:22-48
 *   handle_skewed_data                src/skewed_data_handler.cuh:59-91
 *   shared_memory_hash_join           src/partitioned_join.cuh:178-251
 *   inner_join_cpu (output contract)  src/inner_join_cpu.hpp:24-107
 *
 * Conventions
 *  - Every pointer in a descriptor is a DEVICE pointer unless stated.
 *  - Keys are signed 4- or 8-byte integers (the reference's key_type,
 *    common.cuh:25-39, chosen at run time instead of by -DUSE_8B_KEYS).
 *    Every key value joins, including -1 (the reference's empty-slot
 *    sentinel, hash_join_kernels.cuh:20, which it cannot join).
 *  - Output is a pair of int32 row-index columns (build_row, probe_row), one
 *    entry per matching (build, probe) pair, in no particular order.
 *  - The library never allocates device memory: callers size a workspace
 *    with pj_workspace_size() and pass it in.  Inputs are never modified
 *    (the reference overwrites its inputs in two-pass mode, main.cu:833-838).
 *  - Calls are asynchronous on the given stream (a cudaStream_t; NULL is the
 *    legacy default stream) unless documented as synchronising.  Argument
 *    errors are returned at once; device-side conditions (output capacity,
 *    table overflow, bounded-wait timeout) are recorded in the workspace and
 *    returned by pj_check() after the stream work completes.
 *  - Distinct workspaces may be used concurrently from different threads.
 */
#ifndef PJ_H
#define PJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pj_status {
    PJ_OK = 0,
    PJ_ERR_INVALID = 1,     /* bad argument or unsupported combination */
    PJ_ERR_CAPACITY = 2,    /* output capacity too small; *count holds the required count */
    PJ_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    PJ_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    PJ_ERR_WORKSPACE = 5,   /* workspace missing, misaligned or too small */
    PJ_ERR_OVERFLOW = 6,    /* a shared-memory table overflowed: the plan was too coarse */
    PJ_ERR_ALIGNMENT = 7,   /* an input column is not 16-byte aligned */
    PJ_ERR_INTERNAL = 8     /* a device-side consistency check failed */
} pj_status;

/* cudaStream_t, kept opaque so that this header needs no CUDA headers. */
typedef void* pj_stream;

/* Digit source for radix partitioning. */
enum {
    PJ_DIGIT_RAW = 0,  /* raw key bits, as the reference: partition_kernels.cuh:168,380 */
    PJ_DIGIT_HASH = 1  /* top bits of MurmurHash3_32(key): robust to key patterns */
};

/* Slot function inside a partition's shared-memory table. */
enum {
    PJ_SLOT_FAST = 0,  /* multiply-high range reduction of the unused hash bits */
    PJ_SLOT_REF = 1    /* abs((int)hash % T), as the reference: hash_join_kernels.cuh:100-101 */
};

/* How a partition whose build side exceeds one table is split over CTAs. */
enum {
    PJ_SPLIT_HASH = 0,     /* by hash bits: each probe row visits one table */
    PJ_SPLIT_POSITION = 1  /* by build-row position, every chunk probes all rows:
                              the reference's skew split, skewed_data_handler.cuh:21-43 */
};

/* One join: build and probe key columns (and optional payload columns). */
typedef struct pj_join_desc {
    const void* build_keys;     /* n_build keys of key_bytes each, 16-byte aligned */
    const void* probe_keys;     /* n_probe keys, 16-byte aligned */
    const void* build_payload;  /* optional (NULL): gathered into pj_output.build_payload_out */
    const void* probe_payload;  /* optional (NULL) */
    int64_t n_build;            /* 0 .. 2^31-1 */
    int64_t n_probe;            /* 0 .. 2^31-1 */
    int32_t key_bytes;          /* 4 or 8 */
    int32_t payload_bytes;      /* 0, 4 or 8 */
    int32_t unique_build_keys;  /* non-zero: each probe row matches at most one build row
                                   (the reference's -u, inner_join_cpu.hpp:41-78) */
    int32_t reserved;
} pj_join_desc;

/* Caller-allocated device output. */
typedef struct pj_output {
    int32_t* build_row;         /* capacity entries */
    int32_t* probe_row;         /* capacity entries */
    int64_t capacity;
    int64_t* count;             /* device int64: number of matches (may exceed capacity) */
    void* build_payload_out;    /* optional: build_payload[build_row[i]] */
    void* probe_payload_out;    /* optional: probe_payload[probe_row[i]] */
} pj_output;

/* Shared-memory table of the join. */
enum {
    PJ_TABLE_BUCKET = 0,  /* build tuples counting-sorted by hash bucket (8 B a tuple) */
    PJ_TABLE_OPEN = 1,    /* the reference's open addressing, linear probing,
                             hash_join_kernels.cuh:19-129 */
    PJ_TABLE_COMPACT = 2, /* bucket order with 4-byte entries (hash fingerprint and
                             index of the build tuple): ~2x the tuples per table;
                             a build range must stay within 65536 tuples */
    PJ_TABLE_EXACT = 3    /* bucket order with entries that hold the build row and
                             the hash bits neither the hash digits nor the bucket
                             fix (4 bytes; 8 with an 8-byte key's low word): with
                             them the entry fixes the key, so a lookup loads no
                             build tuple; needs 2^nb buckets with hash digit
                             bits + nb >= the bits of n_build - 1, so hash digits
                             in practice */
};

/* Most heavy probe keys a plan can name. */
#define PJ_MAX_HEAVY 256

/* Execution plan.  pj_plan_default() fills it from the sizes alone,
 * pj_plan_exact() from device histograms.  Passing NULL to pj_inner_join()
 * uses pj_plan_default(). */
typedef struct pj_plan {
    int32_t passes;             /* radix passes: 1, or 2 (pass 2 splits each pass-1
                                   partition by the next bits2 digit bits, as the
                                   reference's partition_input_tables_pass_two,
                                   partitioned_join.cuh:109-175) */
    int32_t bits1;              /* radix bits of pass 1: 2^bits1 partitions */
    int32_t bits2;              /* radix bits of pass 2 (0 for one pass); the join
                                   sees 2^(bits1+bits2) partitions */
    int32_t digit_mode;         /* PJ_DIGIT_* */
    int32_t table_mode;         /* PJ_TABLE_* */
    int32_t slot_mode;          /* PJ_SLOT_* (PJ_TABLE_OPEN) */
    int32_t split_mode;         /* PJ_SPLIT_* */
    int32_t table_capacity;     /* BUCKET: build tuples one table holds; OPEN: slots */
    int32_t probe_chunk;        /* probe tuples of one join work item (multiple of 16) */
    int32_t wc_tuples;          /* tuples per write-combining buffer of pass 1:
                                   2, 4, 8, 16 or 32 (pass 2 sizes its own) */
    int32_t scatter_ctas_per_sm;/* scatter chunks per SM */
    int32_t hist_split;         /* histogram CTAs per scatter chunk */
    float max_fill;             /* OPEN: target fill (the reference's HASH_TABLE_OCC = 0.5) */
    int32_t flags;              /* reserved, 0 */
    int32_t n_heavy;            /* heavy probe keys below (0: no heavy-key path) */
    int32_t heavy_reserved;     /* 0 */
    int64_t heavy_keys[PJ_MAX_HEAVY]; /* probe keys matched outside the partitions, by a
                                   table every CTA holds (unique build keys only);
                                   the reference's skewed_data_handler.cuh:21-91 instead
                                   splits the oversized partitions they cause */
} pj_plan;

/* Human-readable text of a status. */
const char* pj_status_string(pj_status s);

/* Library version string. */
const char* pj_version(void);

/* Plan from the sizes alone (no device work, no synchronisation).  Mirrors
 * the reference's static choice of -n/-N/-f (main.cu:239-251,867) with
 * B200 shared-memory limits. */
pj_status pj_plan_default(const pj_join_desc* desc, pj_plan* plan);

/* The reference's own partitioning flags as a plan: -n partitions_1,
 * -R -N partitions_2 (0: one pass) and -f factor (main.cu:239-251; pass one
 * main.cu:804-810, pass two :826-852, the factor :867).  Pass 1 takes raw
 * key bits as its digit (partition_kernels.cuh:168), pass 2 the top hash
 * bits; partitions are cut into build pieces of at most
 * ceil(factor * n_build / partitions) rows by position, as
 * handle_skewed_data does (skewed_data_handler.cuh:59-91), each piece one
 * BUCKET table.  PJ_ERR_INVALID for partition counts that are not powers of
 * two, a non-positive factor, or a fan-out one scatter pass cannot make. */
pj_status pj_plan_radix(const pj_join_desc* desc, int32_t partitions_1, int32_t partitions_2, float factor,
                        pj_plan* plan);

/* Bytes of device workspace that pj_inner_join / pj_join_count need for
 * this join and plan (plan NULL: the default plan).  The workspace must be
 * 256-byte aligned. */
pj_status pj_workspace_size(const pj_join_desc* desc, const pj_plan* plan, size_t* bytes);

/* Exact-histogram planner: histograms both key columns on the device,
 * reads the histograms back (SYNCHRONISES the stream) and returns a plan in
 * which every partition's table fits shared memory.  Replaces the
 * reference's fixed -n/-N choice and handle_skewed_data's sizing
 * (skewed_data_handler.cuh:59-91). */
pj_status pj_plan_exact(const pj_join_desc* desc, void* workspace, size_t workspace_bytes,
                        pj_plan* plan, pj_stream stream);

/* The join: partition both sides, build and probe per partition, write
 * (build_row, probe_row) pairs.  Replaces main.cu:762-892.  Asynchronous;
 * call pj_check() to learn device-side conditions. */
pj_status pj_inner_join(const pj_join_desc* desc, const pj_plan* plan, pj_output* out,
                        void* workspace, size_t workspace_bytes, pj_stream stream);

/* Number of matching pairs only (written to *count_dev, a device int64);
 * the count the reference takes from its CPU run (main.cu:697-704). */
pj_status pj_join_count(const pj_join_desc* desc, const pj_plan* plan, int64_t* count_dev,
                        void* workspace, size_t workspace_bytes, pj_stream stream);

/* Stage timers of pj_inner_join, like the reference's per-stage cudaEvent
 * timers and CSV columns (main.cu:769-896, 918-948). */
enum {
    PJ_STAGE_BUILD_HIST = 0,     /* pass one of the build side: histogram, */
    PJ_STAGE_BUILD_SCAN = 1,     /*   scan, */
    PJ_STAGE_BUILD_SCATTER = 2,  /*   scatter */
    PJ_STAGE_BUILD_PASS2 = 3,    /* pass two of the build side (empty for one-pass plans) */
    PJ_STAGE_PROBE_HIST = 4,
    PJ_STAGE_PROBE_SCAN = 5,
    PJ_STAGE_PROBE_SCATTER = 6,
    PJ_STAGE_PROBE_PASS2 = 7,
    PJ_STAGE_JOIN_PLAN = 8,      /* work split: the reference's handle_skewed_data */
    PJ_STAGE_JOIN = 9,
    PJ_STAGE_TOTAL = 10,
    PJ_NUM_STAGES = 11
};

/* pj_inner_join with a cudaEvent around every stage; SYNCHRONISES the
 * stream and writes the milliseconds of each stage to stage_ms[PJ_NUM_STAGES]. */
pj_status pj_inner_join_timed(const pj_join_desc* desc, const pj_plan* plan, pj_output* out,
                              void* workspace, size_t workspace_bytes, pj_stream stream,
                              float* stage_ms);

/* pj_inner_join recording events[i] (a cudaEvent_t, created by the caller)
 * on the stream at the start of stage i and events[PJ_STAGE_TOTAL] at the
 * end; asynchronous.  Lets a caller time every kernel inside a timed loop. */
pj_status pj_inner_join_events(const pj_join_desc* desc, const pj_plan* plan, pj_output* out,
                               void* workspace, size_t workspace_bytes, pj_stream stream,
                               void* const* events);

/* SYNCHRONISES the stream and returns the device-side status of the last
 * call that used this workspace (PJ_OK, PJ_ERR_CAPACITY, PJ_ERR_OVERFLOW,
 * PJ_ERR_TIMEOUT or PJ_ERR_INTERNAL), then clears it. */
pj_status pj_check(void* workspace, pj_stream stream);

/* Diagnostics of the bounded device waits (no reference counterpart: the
 * reference's only bounded loop is the build insert's attempt counter,
 * hash_join_kernels.cuh:104-127).  Runs the build side's decoupled
 * look-back scan in the workspace of (desc, plan) with the publish of tile
 * `withhold_tile` withheld, so the tiles after it poll at most
 * `spin_limit` times and give up.  pj_check then returns PJ_ERR_TIMEOUT;
 * the context stays usable and the next join on the workspace starts
 * clean.  Needs withhold_tile + 1 < the scan's tile count (4096 counters
 * a tile); asynchronous. */
pj_status pj_diag_scan_timeout(const pj_join_desc* desc, const pj_plan* plan, void* workspace,
                               size_t workspace_bytes, int64_t withhold_tile, uint32_t spin_limit,
                               pj_stream stream);

/* Size of the library's built-in workspace on each device (64 MiB). */
#define PJ_NOALLOC_SCRATCH_BYTES (64u << 20)

/* pj_inner_join for callers that cannot allocate device memory: no
 * counterpart in the reference, which allocates its buffers itself.  The
 * workspace is a fixed array of PJ_NOALLOC_SCRATCH_BYTES inside the library,
 * one per device, so a caller passes only its key and output columns.  Meant
 * for hosts that bind the join through an FFI without a device allocator, and
 * for callers that must avoid cudaMalloc/cudaFree (cudaFree waits for the
 * whole device).
 * - Joins whose pj_workspace_size() exceeds PJ_NOALLOC_SCRATCH_BYTES (about
 *   2^20 x 2^22 4-byte keys with the default plan) return PJ_ERR_WORKSPACE
 *   before any device work; use pj_inner_join for them.
 * - The first call on each device sets up the array's address (and loads its
 *   module); make it before any stream capture on that device.
 * - Nothing has to be zeroed beforehand: every call clears what it uses.
 * - SYNCHRONISES the stream and returns the final status (that of pj_check).
 * - Calls that overlap in time on one device share the array and race:
 *   serialise them. */
pj_status pj_inner_join_noalloc(const pj_join_desc* desc, const pj_plan* plan, pj_output* out,
                                pj_stream stream);

/* ---- stage entry points (each replaces one reference stage) ------------- */

/* MurmurHash3_32 (seed 0) of every key: MurmurHash3_32<K>::operator(),
 * hash_functions.cuh:80-119.  out: n uint32 (device). */
pj_status pj_hash_keys(const void* keys, int64_t n, int32_t key_bytes, uint32_t* out,
                       pj_stream stream);

/* Table slot of every key for a table of table_slots slots under
 * slot_mode (PJ_SLOT_REF = hash_join_kernels.cuh:100-101).  For
 * PJ_SLOT_FAST, skip_bits top hash bits are treated as already consumed by
 * partition digits.  out: n int32 (device). */
pj_status pj_hash_slots(const void* keys, int64_t n, int32_t key_bytes, int32_t table_slots,
                        int32_t slot_mode, int32_t skip_bits, int32_t* out, pj_stream stream);

/* Global digit histogram in one read of the keys: the reference's
 * histogram_pass_one (partition_kernels.cuh:141-194) for which == 1,
 * histogram_pass_two's global sum (:329-406) for which == 2 and
 * combined_histogram_pass / big_histogram (:86-124, partitioned_join.cuh:22-48)
 * for which == 0 (all bits1+bits2 digit bits).  hist: 2^bits int32 (device),
 * overwritten. */
pj_status pj_radix_histogram(const void* keys, int64_t n, int32_t key_bytes, int32_t digit_mode,
                             int32_t bits1, int32_t bits2, int32_t which, int32_t* hist,
                             pj_stream stream);

/* Radix-partitions one key column into `tuples` (device, capacity
 * pj_partitioned_capacity() tuples) with partition p occupying tuples
 * [offsets[p], offsets[p+1]) (offsets: device int64, 2^(bits1+bits2)+1).
 * A tuple is {uint32 murmur(key), int32 row} for 4-byte keys (the hash is a
 * bijection of the key) and {int32 key_lo, int32 key_hi, uint32 murmur(key),
 * int32 row} for 8-byte keys; padding tuples carry row = -1.
 * Replaces partition_input_tables_pass_one / _pass_two
 * (partitioned_join.cuh:51-175). */
pj_status pj_partition(const void* keys, int64_t n, int32_t key_bytes, const pj_plan* plan,
                       void* tuples, int64_t* offsets, void* workspace, size_t workspace_bytes,
                       pj_stream stream);

/* ---- batches of joins (no reference counterpart: the reference runs one
 * join per process) --------------------------------------------------------
 * Joins whose build side fits one shared-memory table skip partitioning: one
 * persistent kernel drains a (join, probe chunk) work queue over all of
 * them, writing each join's pairs densely to its own output.  Larger joins
 * (up to 2^10 partitions each) are partitioned together -- one histogram,
 * one scan and one scatter launch over both key columns of all of them --
 * and joined by one persistent launch that drains a (join, partition, probe
 * chunk) queue, each match written at an exact position of its join's
 * output.  Wider joins run the partitioned path one after another.  All
 * joins of a batch have the same key width. */
typedef struct pj_batch_config {
    int32_t direct_threads;    /* threads per CTA of the direct kernel: 256, 512 or 1024 */
    int32_t direct_chunk;      /* probe rows per direct work item (>= 1024) */
    int32_t direct_max_build;  /* joins with at most this many build rows go direct (<= 40960) */
    int32_t large_bits_delta;  /* added to the default radix bits of the partitioned joins */
    int32_t large_batched;     /* 1: partitioned joins run together (above); 0: one after another */
} pj_batch_config;

/* Defaults for a key width. */
pj_status pj_batch_config_default(int32_t key_bytes, pj_batch_config* cfg);

/* Workspace bytes for the batch under cfg (NULL: defaults). */
pj_status pj_batch_workspace_size(const pj_join_desc* descs, int32_t n, const pj_batch_config* cfg,
                                  size_t* bytes);

/* Writes the batch's work table into the workspace (SYNCHRONISES).  Call it
 * again whenever descs, outs or cfg change. */
pj_status pj_batch_prepare(const pj_join_desc* descs, const pj_output* outs, int32_t n,
                           const pj_batch_config* cfg, void* workspace, size_t workspace_bytes,
                           pj_stream stream);

/* Runs every join of a prepared batch; outs[i] receives join i's pairs and
 * count.  Asynchronous and free of host synchronisation, so it can be
 * captured in a CUDA graph and replayed.  Device conditions of any join
 * (capacity, overflow) come back from pj_batch_check. */
pj_status pj_join_batch(const pj_join_desc* descs, const pj_output* outs, int32_t n, const pj_batch_config* cfg,
                        void* workspace, size_t workspace_bytes, pj_stream stream);

/* SYNCHRONISES; returns and clears the batch's device status. */
pj_status pj_batch_check(void* workspace, pj_stream stream);

/* Autotuner: times candidate configurations on this batch (where the
 * direct path ends, the direct kernel's block size and chunk, the radix
 * width of the partitioned joins, whether they run together) and returns the
 * fastest in *best (and its
 * time, optional).  SYNCHRONISES; runs the batch many times.  The workspace
 * must hold pj_batch_workspace_size for direct_max_build = 0. */
pj_status pj_batch_autotune(const pj_join_desc* descs, const pj_output* outs, int32_t n, void* workspace,
                            size_t workspace_bytes, pj_stream stream, pj_batch_config* best, float* best_ms);

/* ---- learned planner (no reference counterpart) ----------------------------
 * A small MLP ranks PJ_PLAN_CANDIDATES schedules of a join -- one radix
 * pass with BUCKET, COMPACT or EXACT tables x radix bits (the layout's own
 * width -1, 0, +1) x heavy-key set (none, every heavy key of the probe
 * sample, its 16 most frequent), two radix passes with BUCKET tables at
 * the width +0 and +1, and the exact-histogram planner's own plan
 * (PJ_PLAN_CANDIDATE_EXACT) -- from a sketch of a probe-key sample and the
 * sizes.  It only
 * chooses the schedule: results are those of any plan, and a choice that
 * overflows a table on the device is rerun with pj_plan_exact by the caller
 * (PJ_ERR_OVERFLOW from pj_check). */
#define PJ_MLP_FEATURES 32
#define PJ_MLP_HIDDEN 64
#define PJ_PLAN_CANDIDATES 30
#define PJ_PLAN_CANDIDATE_EXACT 29  /* the last candidate: pj_plan_exact's plan */

/* Shape of an MLP: in -> h1 (ReLU) -> h2 (ReLU) -> out.  Parameters are one
 * float vector W1[in][h1], b1, W2[h1][h2], b2, W3[h2][out], b3. */
typedef struct pj_mlp_dims {
    int32_t in, h1, h2, out;
} pj_mlp_dims;

/* Number of parameters (floats), or -1. */
int64_t pj_mlp_param_count(const pj_mlp_dims* dims);

/* y[batch][out] = MLP(x[batch][in]); acts (batch x (2 h1 + 2 h2) floats)
 * receives the hidden activations for pj_mlp_backward.  Device pointers. */
pj_status pj_mlp_forward(const float* params, const pj_mlp_dims* dims, const float* x, int32_t batch, float* acts,
                         float* y, pj_stream stream);

/* grad (param_count floats) = d(loss)/d(params) given dy = d(loss)/dy of a
 * forward pass on x with activations acts; scratch: batch x (h1 + h2)
 * floats.  Device pointers. */
pj_status pj_mlp_backward(const float* params, const pj_mlp_dims* dims, const float* x, const float* acts,
                          const float* dy, int32_t batch, float* grad, float* scratch, pj_stream stream);

/* Masked mean squared error of y against target (mask NULL: all ones):
 * dy and the loss (device float, optional).  Device pointers. */
pj_status pj_mlp_mse_grad(const float* y, const float* target, const float* mask, int64_t n, float* dy, float* loss,
                          pj_stream stream);

/* One Adam step (step counts from 1).  Device pointers. */
pj_status pj_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t n, float lr, float beta1,
                      float beta2, float eps, int32_t step, pj_stream stream);

/* The planner's input: PJ_MLP_FEATURES floats (host) from a sample of the
 * probe keys (1 % of the rows, 4 096 .. 65 536), and, if heavy is not NULL,
 * the sample's heavy keys (heavy->n_heavy, heavy->heavy_keys).  The
 * workspace is that of the default plan.  SYNCHRONISES. */
pj_status pj_plan_features(const pj_join_desc* desc, void* workspace, size_t workspace_bytes, float* features,
                           pj_plan* heavy, pj_stream stream);

/* Candidate schedule c (0 .. PJ_PLAN_CANDIDATES-1) from the sizes and a heavy
 * set (from pj_plan_features; NULL: none).  PJ_ERR_INVALID if c cannot be
 * built for this join, and for PJ_PLAN_CANDIDATE_EXACT, which needs the
 * device (pj_plan_exact). */
pj_status pj_plan_candidate(const pj_join_desc* desc, int32_t candidate, const pj_plan* heavy, pj_plan* plan);

/* Learned plan: features, the MLP (params: device, PJ_MLP_FEATURES ->
 * PJ_MLP_HIDDEN -> PJ_MLP_HIDDEN -> PJ_PLAN_CANDIDATES, outputs = predicted
 * log2 milliseconds), and the best-ranked candidate that can be built.
 * scores (host, PJ_PLAN_CANDIDATES floats, optional) receives the network's
 * outputs.  SYNCHRONISES. */
pj_status pj_plan_learned(const pj_join_desc* desc, const float* params, void* workspace, size_t workspace_bytes,
                          pj_plan* plan, float* scores, pj_stream stream);

/* Seeded input tables generated on the device: the reference's
 * generate_input_tables (generate_input_tables.cuh:143-226) and its Zipf
 * generator (generate_zipf_input.cuh:50-134).  Build keys lie in
 * [0, rand_max] (distinct when unique_build_keys, which needs
 * rand_max + 1 >= n_build); each probe key is a build key with probability
 * selectivity -- uniformly chosen, or by a Zipf(zipf_theta) law over a
 * seeded rank order when zipf_theta > 0 -- and otherwise a value no build
 * row holds (for repeated build keys: a value above rand_max).  Every value
 * is a pure function of (seed, row).  *hits_dev (device int64, optional)
 * receives the number of probe rows drawn from the build side.
 * Asynchronous. */
pj_status pj_generate_tables(void* build_keys, int64_t n_build, void* probe_keys, int64_t n_probe,
                             int32_t key_bytes, int64_t rand_max, double selectivity, int32_t unique_build_keys,
                             double zipf_theta, uint64_t seed, int64_t* hits_dev, pj_stream stream);

/* Capacity in tuples that pj_partition needs for n keys under plan. */
pj_status pj_partitioned_capacity(int64_t n, int32_t key_bytes, const pj_plan* plan,
                                  int64_t* tuples);

#ifdef __cplusplus
}
#endif

#endif /* PJ_H */
