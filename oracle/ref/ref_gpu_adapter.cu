// ref_gpu_adapter.cu -- drives the reference's own GPU join path on given
// input columns and returns its output records.
//
// TEST INFRASTRUCTURE ONLY (a second, independent checker).  Compiled by
// oracle/build_ref.sh against the unmodified reference headers
// (src/partitioned_join.cuh, src/skewed_data_handler.cuh and what they
// include) into oracle/_ref/libref_gpu_k4.so and, with -DUSE_8B_KEYS,
// libref_gpu_k8.so.  The stage sequence below follows main.cu:762-892
// (main.txt:516-641): optional combined histogram, partition pass one,
// optional pass two (with handle_skewed_data), handle_skewed_data for the
// join, shared_memory_hash_join.  Buffers are allocated here the way
// main.cu allocates them, except that the skew index arrays are sized from
// the actual block count instead of main.cu's fixed over-allocation, so a
// skewed input cannot run past them.
//
// The caller passes HOST arrays; the adapter copies them to the device
// (the reference overwrites its input columns in radix mode), runs the
// stages, and copies the joined records back.  Returns 0 on success,
// a negative code if the configuration is outside the reference's limits
// (each check names the reference line that imposes it), or a positive
// CUDA error code.
#include <cstdint>
#include <cstdio>
#include <cmath>
#include <vector>
#include <algorithm>

#include <cub/cub.cuh>
#include "hash_functions.cuh"
#include "common.cuh"
#include "partitioned_join.cuh"
#include "skewed_data_handler.cuh"

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

#define ADAPTER_TRY(call)                                   \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return static_cast<int>(e_); \
    } while (0)

template <typename T>
int dev_alloc(DevBuf& b, size_t count)
{
    size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    ADAPTER_TRY(cudaMalloc(&b.p, bytes));
    ADAPTER_TRY(cudaMemset(b.p, 0, bytes));
    return 0;
}

bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

}  // namespace

extern "C" {

int ref_gpu_key_bytes(void) { return static_cast<int>(sizeof(key_type)); }

// out_x / out_y receive the .x (key) and .y (probe value, or 0) fields of
// the first `capacity` joined records; *out_count the number written by the
// kernels; stage_ms[0..5] = combined histo, P1, P2, skew, join, total (ms),
// timed as main.cu:769-896 does.
int ref_gpu_partitioned_join(const key_type* build_h, int n_build, const key_type* probe_h,
                             int n_probe, const value_type* build_val_h,
                             const value_type* probe_val_h, int uniq_build_keys, int radix,
                             int num_partitions_1, int num_partitions_2,
                             float max_partition_size_factor, int combined_histo,
                             int joined_capacity, key_type* out_x, value_type* out_y,
                             int* out_count, float* stage_ms)
{
    const bool with_value = build_val_h != nullptr && probe_val_h != nullptr;
    if (!is_pow2(num_partitions_1) || (radix && !is_pow2(num_partitions_2))) return -1;  // main.cu:239-251
    if (num_partitions_1 > 1024 || (radix && num_partitions_2 > 1024)) return -2;        // BlockScan 512x2, partition_kernels.cuh:21,261-274
    if (combined_histo && sizeof(key_type) != 4) return -3;                              // main.cu:211-216
    if (n_build <= 0 || n_probe <= 0 || joined_capacity <= 0) return -4;

    const int num_bits_2 = radix ? static_cast<int>(std::log2(num_partitions_2)) : 0;
    const int num_partitions = radix ? num_partitions_1 * num_partitions_2 : num_partitions_1;
    const int num_unroll = with_value ? N_UNROLL_W_VAL : N_UNROLL;

    // Shared memory of the join kernel must fit the 96 000 B attribute
    // (partitioned_join.cuh:198-199,324); otherwise the reference launch fails.
    const int base_build_tbl_size_each_part =
        static_cast<int>(std::ceil(max_partition_size_factor * n_build / num_partitions));
    const long long hash_table_size = static_cast<long long>(std::ceil(1.0 * base_build_tbl_size_each_part / HASH_TABLE_OCC));
    const long long out_smem = static_cast<long long>(std::ceil(1.0 * joined_capacity / num_partitions));
    if (hash_table_size * (long long)sizeof(hash_map_type) + out_smem * (long long)sizeof(joined_type) > 96000) return -5;

    DevBuf build_tbl, probe_tbl, build_tbl_p, probe_tbl_p, build_val, probe_val, build_val_p, probe_val_p;
    if (int e = dev_alloc<key_type>(build_tbl, n_build)) return e;
    if (int e = dev_alloc<key_type>(probe_tbl, n_probe)) return e;
    if (int e = dev_alloc<key_type>(build_tbl_p, n_build)) return e;
    if (int e = dev_alloc<key_type>(probe_tbl_p, n_probe)) return e;
    ADAPTER_TRY(cudaMemcpy(build_tbl.p, build_h, sizeof(key_type) * n_build, cudaMemcpyHostToDevice));
    ADAPTER_TRY(cudaMemcpy(probe_tbl.p, probe_h, sizeof(key_type) * n_probe, cudaMemcpyHostToDevice));
    if (with_value) {
        if (int e = dev_alloc<value_type>(build_val, n_build)) return e;
        if (int e = dev_alloc<value_type>(probe_val, n_probe)) return e;
        if (int e = dev_alloc<value_type>(build_val_p, n_build)) return e;
        if (int e = dev_alloc<value_type>(probe_val_p, n_probe)) return e;
        ADAPTER_TRY(cudaMemcpy(build_val.p, build_val_h, sizeof(value_type) * n_build, cudaMemcpyHostToDevice));
        ADAPTER_TRY(cudaMemcpy(probe_val.p, probe_val_h, sizeof(value_type) * n_probe, cudaMemcpyHostToDevice));
    }

    DevBuf build_histo, probe_histo, build_histo_s, probe_histo_s;
    DevBuf build_histo_p2, probe_histo_p2, build_histo_s_p2, probe_histo_s_p2;
    if (int e = dev_alloc<size_type>(build_histo, num_partitions_1)) return e;
    if (int e = dev_alloc<size_type>(probe_histo, num_partitions_1)) return e;
    if (int e = dev_alloc<size_type>(build_histo_s, num_partitions_1)) return e;
    if (int e = dev_alloc<size_type>(probe_histo_s, num_partitions_1)) return e;
    if (radix) {
        if (int e = dev_alloc<size_type>(build_histo_p2, num_partitions)) return e;
        if (int e = dev_alloc<size_type>(probe_histo_p2, num_partitions)) return e;
        if (int e = dev_alloc<size_type>(build_histo_s_p2, num_partitions)) return e;
        if (int e = dev_alloc<size_type>(probe_histo_s_p2, num_partitions)) return e;
    }

    // Skew index arrays.  Block counts are bounded by partitions + rows/chunk
    // (get_number_of_blocks_each_partition, skewed_data_handler.cuh:21-43);
    // +2 covers populate_index_array's write at the scanned total (:46-56).
    const int p2_chunk = BLOCK_SIZE_PARTITION * num_unroll;
    const long long p2_blocks_build = num_partitions_1 + n_build / p2_chunk + 2;
    const long long p2_blocks_probe = num_partitions_1 + n_probe / p2_chunk + 2;
    const long long join_blocks = num_partitions + n_build / std::max(1, base_build_tbl_size_each_part) + 2;
    DevBuf pi_p2_b, pia_p2_b, pi_p2_p, pia_p2_p, nb_p2_b, nbs_p2_b, nb_p2_p, nbs_p2_p;
    DevBuf partition_index, partition_index_alt, nb_join, nbs_join;
    if (radix) {
        if (int e = dev_alloc<size_type>(pi_p2_b, p2_blocks_build)) return e;
        if (int e = dev_alloc<size_type>(pia_p2_b, p2_blocks_build)) return e;
        if (int e = dev_alloc<size_type>(pi_p2_p, p2_blocks_probe)) return e;
        if (int e = dev_alloc<size_type>(pia_p2_p, p2_blocks_probe)) return e;
        if (int e = dev_alloc<size_type>(nb_p2_b, num_partitions_1 + 1)) return e;
        if (int e = dev_alloc<size_type>(nbs_p2_b, num_partitions_1 + 1)) return e;
        if (int e = dev_alloc<size_type>(nb_p2_p, num_partitions_1 + 1)) return e;
        if (int e = dev_alloc<size_type>(nbs_p2_p, num_partitions_1 + 1)) return e;
    }
    if (int e = dev_alloc<size_type>(partition_index, join_blocks)) return e;
    if (int e = dev_alloc<size_type>(partition_index_alt, join_blocks)) return e;
    if (int e = dev_alloc<size_type>(nb_join, num_partitions + 1)) return e;
    if (int e = dev_alloc<size_type>(nbs_join, num_partitions + 1)) return e;

    DevBuf joined, global_index;
    if (int e = dev_alloc<joined_type>(joined, joined_capacity)) return e;
    if (int e = dev_alloc<size_type>(global_index, 1)) return e;

    // CUB temporary storage: the maximum over every scan the stages run (main.txt:491-510).
    size_t temp_bytes = 0, t = 0;
    size_type* sp = nullptr;
    cub::DeviceScan::ExclusiveSum(nullptr, t, sp, sp, num_partitions_1); temp_bytes = std::max(temp_bytes, t);
    cub::DeviceScan::ExclusiveSum(nullptr, t, sp, sp, num_partitions); temp_bytes = std::max(temp_bytes, t);
    cub::DeviceScan::InclusiveSum(nullptr, t, sp, sp, num_partitions + 1); temp_bytes = std::max(temp_bytes, t);
    cub::DeviceScan::InclusiveSum(nullptr, t, sp, sp, num_partitions_1 + 1); temp_bytes = std::max(temp_bytes, t);
    cub::DeviceScan::InclusiveSum(nullptr, t, sp, sp, (int)std::max({p2_blocks_build, p2_blocks_probe, join_blocks})); temp_bytes = std::max(temp_bytes, t);
    DevBuf temp;
    if (int e = dev_alloc<char>(temp, temp_bytes)) return e;

    int* num_block_join_h = nullptr;
    int* num_block_p2_build_h = nullptr;
    int* num_block_p2_probe_h = nullptr;
    ADAPTER_TRY(cudaMallocHost(&num_block_join_h, sizeof(int)));
    ADAPTER_TRY(cudaMallocHost(&num_block_p2_build_h, sizeof(int)));
    ADAPTER_TRY(cudaMallocHost(&num_block_p2_probe_h, sizeof(int)));

    set_shared_memory_config(uniq_build_keys != 0, with_value);

    cudaEvent_t start, stop;
    ADAPTER_TRY(cudaEventCreate(&start));
    ADAPTER_TRY(cudaEventCreate(&stop));
    float combined_ms = 0, p1_ms = 0, p2_ms = 0, skew_ms = 0, join_ms = 0;

    auto K = [](DevBuf& b) { return static_cast<key_type*>(b.p); };
    auto V = [](DevBuf& b) { return static_cast<value_type*>(b.p); };
    auto S = [](DevBuf& b) { return static_cast<size_type*>(b.p); };

    size_type* join_build_global_histo = radix ? S(build_histo_p2) : S(build_histo);
    size_type* join_probe_global_histo = radix ? S(probe_histo_p2) : S(probe_histo);

    if (combined_histo) {
        cudaEventRecord(start, 0);
        combined_histogram_pass(join_build_global_histo, S(build_histo), K(build_tbl), n_build,
                                num_partitions, num_partitions_1, num_partitions_2, radix != 0);
        combined_histogram_pass(join_probe_global_histo, S(probe_histo), K(probe_tbl), n_probe,
                                num_partitions, num_partitions_1, num_partitions_2, radix != 0);
        cudaEventRecord(stop, 0);
        cudaEventSynchronize(stop);
        cudaEventElapsedTime(&combined_ms, start, stop);
    }

    cudaEventRecord(start, 0);
    partition_input_tables_pass_one<key_type, size_type, value_type>(
        K(build_tbl_p), V(build_val_p), S(build_histo), S(build_histo_s), num_partitions_1, K(build_tbl),
        V(build_val), n_build, num_partitions_1, temp.p, temp_bytes, with_value, num_bits_2, combined_histo != 0);
    partition_input_tables_pass_one<key_type, size_type, value_type>(
        K(probe_tbl_p), V(probe_val_p), S(probe_histo), S(probe_histo_s), num_partitions_1, K(probe_tbl),
        V(probe_val), n_probe, num_partitions_1, temp.p, temp_bytes, with_value, num_bits_2, combined_histo != 0);
    cudaEventRecord(stop, 0);
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&p1_ms, start, stop);

    if (radix) {
        cudaEventRecord(start, 0);
        handle_skewed_data<size_type>(S(build_histo), n_build, p2_chunk, num_partitions_1, S(pi_p2_b),
                                      S(pia_p2_b), S(nb_p2_b), S(nbs_p2_b), num_block_p2_build_h, temp.p,
                                      temp_bytes);
        partition_input_tables_pass_two<key_type, size_type, value_type>(
            K(build_tbl), V(build_val), S(build_histo_p2), S(build_histo_s_p2), num_partitions, K(build_tbl_p),
            V(build_val_p), n_build, num_partitions_1, num_partitions_2, S(nbs_p2_b), S(pi_p2_b),
            *num_block_p2_build_h, temp.p, temp_bytes, S(build_histo), with_value, combined_histo != 0);
        handle_skewed_data<size_type>(S(probe_histo), n_probe, p2_chunk, num_partitions_1, S(pi_p2_p),
                                      S(pia_p2_p), S(nb_p2_p), S(nbs_p2_p), num_block_p2_probe_h, temp.p,
                                      temp_bytes);
        partition_input_tables_pass_two<key_type, size_type, value_type>(
            K(probe_tbl), V(probe_val), S(probe_histo_p2), S(probe_histo_s_p2), num_partitions, K(probe_tbl_p),
            V(probe_val_p), n_probe, num_partitions_1, num_partitions_2, S(nbs_p2_p), S(pi_p2_p),
            *num_block_p2_probe_h, temp.p, temp_bytes, S(probe_histo), with_value, combined_histo != 0);
        cudaEventRecord(stop, 0);
        cudaEventSynchronize(stop);
        cudaEventElapsedTime(&p2_ms, start, stop);
    }

    cudaEventRecord(start, 0);
    key_type* join_build_tbl = radix ? K(build_tbl) : K(build_tbl_p);
    key_type* join_probe_tbl = radix ? K(probe_tbl) : K(probe_tbl_p);
    value_type* join_build_val = radix ? V(build_val) : V(build_val_p);
    value_type* join_probe_val = radix ? V(probe_val) : V(probe_val_p);
    handle_skewed_data<size_type>(join_build_global_histo, n_build, base_build_tbl_size_each_part, num_partitions,
                                  S(partition_index), S(partition_index_alt), S(nb_join), S(nbs_join),
                                  num_block_join_h, temp.p, temp_bytes);
    cudaEventRecord(stop, 0);
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&skew_ms, start, stop);

    cudaEventRecord(start, 0);
    shared_memory_hash_join<key_type, size_type, value_type, joined_type>(
        static_cast<joined_type*>(joined.p), join_build_tbl, join_build_val, n_build, join_probe_tbl, join_probe_val,
        n_probe, base_build_tbl_size_each_part, S(global_index), S(nbs_join), S(partition_index), *num_block_join_h,
        num_partitions, uniq_build_keys != 0, join_build_global_histo, join_probe_global_histo, with_value,
        joined_capacity);
    cudaEventRecord(stop, 0);
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&join_ms, start, stop);
    ADAPTER_TRY(cudaGetLastError());
    ADAPTER_TRY(cudaDeviceSynchronize());

    int count = 0;
    ADAPTER_TRY(cudaMemcpy(&count, global_index.p, sizeof(int), cudaMemcpyDeviceToHost));
    *out_count = count;
    std::vector<joined_type> host(static_cast<size_t>(joined_capacity));
    ADAPTER_TRY(cudaMemcpy(host.data(), joined.p, sizeof(joined_type) * joined_capacity, cudaMemcpyDeviceToHost));
    const int n_out = std::min(count, joined_capacity);
    for (int i = 0; i < n_out; ++i) {
        out_x[i] = host[i].x;
        out_y[i] = host[i].y;
    }
    if (stage_ms) {
        stage_ms[0] = combined_ms;
        stage_ms[1] = p1_ms;
        stage_ms[2] = p2_ms;
        stage_ms[3] = skew_ms;
        stage_ms[4] = join_ms;
        stage_ms[5] = combined_ms + p1_ms + p2_ms + skew_ms + join_ms;  // main.cu:895-896
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    cudaFreeHost(num_block_join_h);
    cudaFreeHost(num_block_p2_build_h);
    cudaFreeHost(num_block_p2_probe_h);
    return 0;
}

}  // extern "C"
