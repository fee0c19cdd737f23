// partitioned_join_cli.cu -- the command-line drop-in for the reference's
// `partitioned_join` binary (main.cu): same options (main.cu:100-188), the
// same settings/results report and the same CSV columns
// (scripts/bench_partitioned_join.sh:13), so the reference's scripts run
// unchanged against it.  The join itself runs through include/pj.h.
//
// What differs, on purpose:
//  * Tables are generated on the device by pj_generate_tables (same recipe
//    as generate_input_tables.cuh; rand_max defaults to twice the default
//    build size, 2^21, as main.cu:79 computes it before parsing).
//  * -n, -R -N and -f plan the join as the reference's flags do
//    (pj_plan_radix: 2^log2(n) first-pass partitions by raw key bits, with -R
//    a second pass into N partitions each, build pieces of at most
//    ceil(f * |R| / partitions) rows).  The second pass splits by hash bits
//    rather than the key's low bits.  Without -n the exact-histogram planner
//    chooses (pj_plan_exact); the reference requires -n.  The CSV columns
//    keep their meaning: "part P1" is the first pass of both sides
//    (histograms, scans, scatters), "part P2" the second pass of both sides,
//    "handle skew" the work split, "join" the build/probe kernel, "total"
//    their sum.  With -H the first pass's histogram time is reported under
//    "combined histo".
//  * The check (without -S) does not re-run the join on the CPU: every
//    output pair is verified on the device (both rows in range and their
//    keys equal), and for unique build keys the pair count must equal the
//    number of probe rows the generator drew from the build side.
//    num errors = bad pairs + |count - expected|.
//  * -F reads raw little-endian key files (-B, -P) of -b and -p keys; the
//    reference's -F loads TPC-H Q4 .tbl files from a fixed path.
//  * -K 8 selects 8-byte keys at run time (the reference: -DUSE_8B_KEYS).
//  * The join runs once untimed, then once timed.
#include <getopt.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pj.h"

namespace {

#define CLI_CUDA(call)                                                                            \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            std::cerr << "CUDA error " << cudaGetErrorString(e_) << " at " << __LINE__ << std::endl; \
            std::exit(1);                                                                         \
        }                                                                                         \
    } while (0)

#define CLI_PJ(call)                                                                              \
    do {                                                                                          \
        pj_status s_ = (call);                                                                    \
        if (s_ != PJ_OK) {                                                                        \
            std::cerr << "Error: " #call ": " << pj_status_string(s_) << std::endl;               \
            std::exit(1);                                                                         \
        }                                                                                         \
    } while (0)

bool is_power_of_two(int x) { return x > 0 && (x & (x - 1)) == 0; }

// Count of output pairs whose rows are out of range or whose keys differ.
template <typename K>
__global__ void verify_pairs_kernel(const int32_t* __restrict__ br, const int32_t* __restrict__ pr, int64_t n,
                                    const K* __restrict__ bk, int64_t nb, const K* __restrict__ pk, int64_t np,
                                    unsigned long long* bad)
{
    unsigned long long mine = 0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t b = br[i], p = pr[i];
        if (b < 0 || b >= nb || p < 0 || p >= np || bk[b] != pk[p]) ++mine;
    }
    if (mine) atomicAdd(bad, mine);
}

struct Options {
    int build_tbl_size = 1 << 20;
    int probe_tbl_size = 1 << 20;
    double selectivity = 0.03;
    int rand_max = (1 << 20) << 1;
    bool uniq_build_tbl_keys = false;
    bool read_from_file = false;
    std::string build_tbl_file, probe_tbl_file;
    int verbosity = 0;
    float max_partition_size_factor = 3.0f;
    bool radix_partition = false;
    int num_partitions_1 = -1, num_partitions_2 = -1;
    bool skip_cpu_run = false;
    int output_size = -1;
    bool with_value = false;
    bool csv = false;
    int skewed_data_mode = 0;
    float zipf_factor = -1.0f;
    bool do_combined_histo_pass = false;
    int key_bytes = 4;
};

void usage()
{
    const char* lines[][3] = {
        {"b", "build_tbl_size [arg]", "Build table size [default: 1048576]"},
        {"p", "probe_tbl_size [arg]", "Probe table size [default: 1048576]"},
        {"s", "selectivity [arg]", "Selectivity [default: 0.030000]"},
        {"r", "rand_max [arg]", "Maximum value of generated data [default: 2097152]"},
        {"u", "uniq_build_tbl_keys", "Unique keys for build table [default: false]"},
        {"F", "read_from_file", "Read raw key files given by -B and -P [default: false]"},
        {"B", "build_tbl_file [arg]", "Build table file path [default: ]"},
        {"P", "probe_tbl_file [arg]", "Probe table file path [default: ]"},
        {"v", "verbosity [arg]", "Verbosity level [default: 0]"},
        {"f", "max_partition_size_factor [arg]", "Max partition size factor [default: 3.000000]"},
        {"R", "radix_partition", "Two-pass radix partition [default: false]"},
        {"n", "num_partitions_1 [arg]", "Number of partitions for pass 1 (none: exact-histogram plan) [default: -1]"},
        {"N", "num_partitions_2 [arg]", "Number of partitions for pass 2 [default: -1]"},
        {"S", "skip_cpu_run [arg]", "Skip the check and give the output size [default: -1]"},
        {"V", "with_value", "Add value columns to input tables [default: false]"},
        {"C", "csv", "Output results in csv format [default: false]"},
        {"Z", "skewed_data_mode [arg]", "Skewed data on [0: none, 1: build, 2: probe, 3: both] [default: 0]"},
        {"z", "zipf_dist [arg]", "Zipf factor for skewed data [0-1] [default: -1.000000]"},
        {"H", "do_combined_histogram_pass", "Report histograms as the combined histogram pass [default: false]"},
        {"K", "key_bytes [arg]", "Key width in bytes, 4 or 8 [default: 4]"},
    };
    std::cout << "Usage:" << std::endl;
    for (auto& l : lines) std::cout << "  -" << l[0] << ", --" << l[1] << std::endl << "    " << l[2] << std::endl;
}

Options parse(int argc, char** argv)
{
    Options o;
    const option long_opts[] = {
        {"build_tbl_size", required_argument, nullptr, 'b'},
        {"probe_tbl_size", required_argument, nullptr, 'p'},
        {"selectivity", required_argument, nullptr, 's'},
        {"rand_max", required_argument, nullptr, 'r'},
        {"uniq_build_tbl_keys", no_argument, nullptr, 'u'},
        {"read_from_file", no_argument, nullptr, 'F'},
        {"build_tbl_file", required_argument, nullptr, 'B'},
        {"probe_tbl_file", required_argument, nullptr, 'P'},
        {"verbosity", required_argument, nullptr, 'v'},
        {"max_partition_size_factor", required_argument, nullptr, 'f'},
        {"radix_partition", no_argument, nullptr, 'R'},
        {"num_partitions_1", required_argument, nullptr, 'n'},
        {"num_partitions_2", required_argument, nullptr, 'N'},
        {"skip_cpu_run", required_argument, nullptr, 'S'},
        {"with_value", no_argument, nullptr, 'V'},
        {"csv", no_argument, nullptr, 'C'},
        {"skewed_data_mode", required_argument, nullptr, 'Z'},
        {"zipf_dist", required_argument, nullptr, 'z'},
        {"do_combined_histogram_pass", no_argument, nullptr, 'H'},
        {"key_bytes", required_argument, nullptr, 'K'},
        {nullptr, 0, nullptr, 0},
    };
    int opt;
    while ((opt = getopt_long(argc, argv, "b:p:s:r:uFB:P:v:f:Rn:N:S:VCZ:z:HhK:", long_opts, nullptr)) != -1) {
        switch (opt) {
        case 'b': o.build_tbl_size = std::atoi(optarg); break;
        case 'p': o.probe_tbl_size = std::atoi(optarg); break;
        case 's': o.selectivity = std::atof(optarg); break;
        case 'r': o.rand_max = std::atoi(optarg); break;
        case 'u': o.uniq_build_tbl_keys = true; break;
        case 'F': o.read_from_file = true; break;
        case 'B': o.build_tbl_file = optarg; break;
        case 'P': o.probe_tbl_file = optarg; break;
        case 'v': o.verbosity = std::atoi(optarg); break;
        case 'f': o.max_partition_size_factor = static_cast<float>(std::atof(optarg)); break;
        case 'R': o.radix_partition = true; break;
        case 'n': o.num_partitions_1 = std::atoi(optarg); break;
        case 'N': o.num_partitions_2 = std::atoi(optarg); break;
        case 'S': o.skip_cpu_run = true; o.output_size = std::atoi(optarg); break;
        case 'V': o.with_value = true; break;
        case 'C': o.csv = true; break;
        case 'Z': o.skewed_data_mode = std::atoi(optarg); break;
        case 'z': o.zipf_factor = static_cast<float>(std::atof(optarg)); break;
        case 'H': o.do_combined_histo_pass = true; break;
        case 'K': o.key_bytes = std::atoi(optarg); break;
        case 'h': usage(); std::exit(EXIT_FAILURE);
        default:
            std::cout << "Please use -h or --help for the list of options" << std::endl;
            std::exit(EXIT_FAILURE);
        }
    }
    return o;
}

template <typename K>
bool read_keys(const std::string& path, std::vector<K>& v, int n)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    v.resize(static_cast<size_t>(n));
    const size_t got = std::fread(v.data(), sizeof(K), v.size(), f);
    std::fclose(f);
    return got == v.size();
}

template <typename K>
int run(Options& o)
{
    // partition-count arguments, validated as main.cu:227-251 does
    if (o.do_combined_histo_pass && sizeof(K) == 8) {
        std::cerr << "Error: combined histo pass is not supported for 8B key. Disable -H." << std::endl;
        return 1;
    }
    int num_bits_1 = 0, num_bits_2 = 0;
    const bool plan_from_flags = o.num_partitions_1 != -1 || o.radix_partition;
    if (!plan_from_flags) {
        // no partition flags: the exact-histogram planner chooses
    } else if (!o.radix_partition && is_power_of_two(o.num_partitions_1)) {
        num_bits_1 = static_cast<int>(std::log2(o.num_partitions_1));
    } else if (o.radix_partition && is_power_of_two(o.num_partitions_1) && is_power_of_two(o.num_partitions_2)) {
        num_bits_1 = static_cast<int>(std::log2(o.num_partitions_1));
        num_bits_2 = static_cast<int>(std::log2(o.num_partitions_2));
    } else {
        std::cerr << "Error: num_partition must be power of two." << std::endl;
        return 1;
    }
    if (o.build_tbl_size < 0 || o.probe_tbl_size < 0) {
        std::cerr << "Error: table sizes must not be negative." << std::endl;
        return 1;
    }
    const int64_t nb = o.build_tbl_size, np = o.probe_tbl_size;
    long long device_memory_used = 0;
    K *build = nullptr, *probe = nullptr;
    CLI_CUDA(cudaMalloc(&build, sizeof(K) * std::max<int64_t>(nb, 1)));
    CLI_CUDA(cudaMalloc(&probe, sizeof(K) * std::max<int64_t>(np, 1)));
    device_memory_used += (nb + np) * sizeof(K);
    int64_t* hits_d = nullptr;
    CLI_CUDA(cudaMalloc(&hits_d, sizeof(int64_t)));
    int64_t hits = -1;
    if (o.read_from_file) {
        if (!o.csv) std::cout << "[*] Reading input tables" << std::endl;
        std::vector<K> hb, hp;
        if (!read_keys(o.build_tbl_file, hb, o.build_tbl_size) || !read_keys(o.probe_tbl_file, hp, o.probe_tbl_size)) {
            std::cerr << "Error: cannot read " << o.build_tbl_size << " and " << o.probe_tbl_size
                      << " keys from -B/-P files." << std::endl;
            return 1;
        }
        CLI_CUDA(cudaMemcpy(build, hb.data(), sizeof(K) * nb, cudaMemcpyHostToDevice));
        CLI_CUDA(cudaMemcpy(probe, hp.data(), sizeof(K) * np, cudaMemcpyHostToDevice));
    } else {
        if (o.skewed_data_mode != 0) {  // main.cu:343-349
            o.selectivity = 1;
            o.uniq_build_tbl_keys = o.skewed_data_mode == 2;
        }
        if (!o.csv) std::cout << "[*] Generating input tables" << std::endl;
        if (o.uniq_build_tbl_keys && static_cast<int64_t>(o.rand_max) + 1 < nb) {
            std::cerr << "Error: unique build keys need rand_max >= build table size - 1." << std::endl;
            return 1;
        }
        CLI_PJ(pj_generate_tables(build, nb, probe, np, sizeof(K), o.rand_max, o.selectivity,
                                  o.uniq_build_tbl_keys ? 1 : 0, 0.0, 1234, hits_d, nullptr));
        CLI_CUDA(cudaMemcpy(&hits, hits_d, sizeof(int64_t), cudaMemcpyDeviceToHost));
    }
    // value columns: the row ids (the reference zero-fills them, main.cu:282-300)
    int32_t *bval = nullptr, *pval = nullptr;
    if (o.with_value) {
        std::vector<int32_t> ids(static_cast<size_t>(std::max<int64_t>(nb, np)));
        for (size_t i = 0; i < ids.size(); ++i) ids[i] = static_cast<int32_t>(i);
        CLI_CUDA(cudaMalloc(&bval, sizeof(int32_t) * std::max<int64_t>(nb, 1)));
        CLI_CUDA(cudaMalloc(&pval, sizeof(int32_t) * std::max<int64_t>(np, 1)));
        CLI_CUDA(cudaMemcpy(bval, ids.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
        CLI_CUDA(cudaMemcpy(pval, ids.data(), sizeof(int32_t) * np, cudaMemcpyHostToDevice));
        device_memory_used += (nb + np) * sizeof(int32_t);
    }

    pj_join_desc d = {};
    d.build_keys = build;
    d.probe_keys = probe;
    d.n_build = nb;
    d.n_probe = np;
    d.key_bytes = sizeof(K);
    d.unique_build_keys = o.uniq_build_tbl_keys ? 1 : 0;
    if (o.with_value) {
        d.build_payload = bval;
        d.probe_payload = pval;
        d.payload_bytes = 4;
    }
    pj_plan plan;
    if (plan_from_flags) {
        const pj_status ps = pj_plan_radix(&d, o.num_partitions_1, o.radix_partition ? o.num_partitions_2 : 0,
                                           o.max_partition_size_factor, &plan);
        if (ps != PJ_OK) {
            std::cerr << "Error: partition flags -n " << o.num_partitions_1 << (o.radix_partition ? " -N " : "")
                      << (o.radix_partition ? std::to_string(o.num_partitions_2) : std::string()) << " -f "
                      << o.max_partition_size_factor << ": " << pj_status_string(ps) << std::endl;
            return 1;
        }
    } else {
        CLI_PJ(pj_plan_default(&d, &plan));
    }
    size_t ws_bytes = 0;
    CLI_PJ(pj_workspace_size(&d, &plan, &ws_bytes));
    void* ws = nullptr;
    CLI_CUDA(cudaMalloc(&ws, ws_bytes));
    if (!plan_from_flags && nb > 0 && np > 0) {
        CLI_PJ(pj_plan_exact(&d, ws, ws_bytes, &plan, nullptr));
        size_t need = 0;
        CLI_PJ(pj_workspace_size(&d, &plan, &need));
        if (need > ws_bytes) {
            CLI_CUDA(cudaFree(ws));
            ws_bytes = need;
            CLI_CUDA(cudaMalloc(&ws, ws_bytes));
        }
    }
    device_memory_used += ws_bytes;

    // output capacity: -S, else the device count
    int64_t* count_d = nullptr;
    CLI_CUDA(cudaMalloc(&count_d, sizeof(int64_t)));
    int64_t joined_size = 0;
    if (o.skip_cpu_run) {
        joined_size = std::max(o.output_size, 0);
    } else {
        CLI_PJ(pj_join_count(&d, &plan, count_d, ws, ws_bytes, nullptr));
        CLI_PJ(pj_check(ws, nullptr));
        CLI_CUDA(cudaMemcpy(&joined_size, count_d, sizeof(int64_t), cudaMemcpyDeviceToHost));
    }
    int32_t *br = nullptr, *pr = nullptr, *bvo = nullptr, *pvo = nullptr;
    const int64_t cap = std::max<int64_t>(joined_size, 1);
    CLI_CUDA(cudaMalloc(&br, sizeof(int32_t) * cap));
    CLI_CUDA(cudaMalloc(&pr, sizeof(int32_t) * cap));
    device_memory_used += 2 * cap * sizeof(int32_t);
    if (o.with_value) {
        CLI_CUDA(cudaMalloc(&bvo, sizeof(int32_t) * cap));
        CLI_CUDA(cudaMalloc(&pvo, sizeof(int32_t) * cap));
        device_memory_used += 2 * cap * sizeof(int32_t);
    }
    pj_output out = {br, pr, joined_size, count_d, bvo, pvo};

    // settings line / report, as main.cu:420-470
    if (o.csv) {
        const int tuple_byte = o.with_value ? static_cast<int>(sizeof(K) + sizeof(int32_t)) : static_cast<int>(sizeof(K));
        std::cout << o.build_tbl_size << "," << o.probe_tbl_size << "," << sizeof(K) << "," << tuple_byte << ","
                  << o.selectivity << "," << o.uniq_build_tbl_keys << "," << o.num_partitions_1 << ","
                  << o.num_partitions_2 << "," << o.max_partition_size_factor << "," << o.skewed_data_mode << ","
                  << o.zipf_factor << ",";
    } else {
        std::cout << "[*] Settings:" << std::endl;
        std::cout << "    build tabel size     = " << o.build_tbl_size << std::endl;
        std::cout << "    probe tabel size     = " << o.probe_tbl_size << std::endl;
        std::cout << "    has value col        = " << std::boolalpha << o.with_value << std::endl;
        std::cout << "    skewed data mode     = " << o.skewed_data_mode << std::endl;
        if (o.skewed_data_mode != 0) std::cout << "    zipf factor          = " << o.zipf_factor << std::endl;
        if (o.read_from_file) {
            std::cout << "    build table path     = " << o.build_tbl_file << std::endl;
            std::cout << "    probe table path     = " << o.probe_tbl_file << std::endl;
        } else {
            std::cout << "    selectivity          = " << o.selectivity << std::endl;
            std::cout << "    rand max             = " << o.rand_max << std::endl;
        }
        std::cout << "    uniq build tbl keys  = " << std::boolalpha << o.uniq_build_tbl_keys << std::endl;
        std::cout << "    max part size factor = " << o.max_partition_size_factor << std::endl;
        std::cout << "    radix partition      = " << std::boolalpha << o.radix_partition << std::endl;
        std::cout << "    num partitions P1    = " << o.num_partitions_1 << std::endl;
        std::cout << "    num bits P1          = " << num_bits_1 << std::endl;
        if (o.radix_partition) {
            std::cout << "    num partitions P2    = " << o.num_partitions_2 << std::endl;
            std::cout << "    num bits P2          = " << num_bits_2 << std::endl;
        }
        std::cout << "    B200 plan            = " << (1 << plan.bits1) << " partitions ("
                  << (plan.digit_mode == PJ_DIGIT_RAW ? "raw key bits" : "hash bits") << ")";
        if (plan.passes == 2) std::cout << " x " << (1 << plan.bits2) << " (hash bits)";
        std::cout << ", "
                  << (plan.table_mode == PJ_TABLE_BUCKET    ? "bucket"
                      : plan.table_mode == PJ_TABLE_COMPACT ? "compact"
                      : plan.table_mode == PJ_TABLE_EXACT   ? "exact"
                                                            : "open")
                  << " tables of " << plan.table_capacity << std::endl;
        std::cout << "[*] Performing join" << std::endl;
    }

    // one untimed run, then the timed one
    float ms[PJ_NUM_STAGES] = {};
    CLI_PJ(pj_inner_join(&d, &plan, &out, ws, ws_bytes, nullptr));
    CLI_PJ(pj_check(ws, nullptr));
    CLI_PJ(pj_inner_join_timed(&d, &plan, &out, ws, ws_bytes, nullptr, ms));
    const pj_status dev_status = pj_check(ws, nullptr);
    if (dev_status != PJ_OK && dev_status != PJ_ERR_CAPACITY) {
        std::cerr << "Error: join: " << pj_status_string(dev_status) << std::endl;
        return 1;
    }
    int64_t count = 0;
    CLI_CUDA(cudaMemcpy(&count, count_d, sizeof(int64_t), cudaMemcpyDeviceToHost));

    const float hist_ms = ms[PJ_STAGE_BUILD_HIST] + ms[PJ_STAGE_PROBE_HIST];
    float partition_one_elapsed_ms = ms[PJ_STAGE_BUILD_HIST] + ms[PJ_STAGE_BUILD_SCAN] + ms[PJ_STAGE_BUILD_SCATTER] +
                                     ms[PJ_STAGE_PROBE_HIST] + ms[PJ_STAGE_PROBE_SCAN] + ms[PJ_STAGE_PROBE_SCATTER];
    float combined_histo_elapsed_ms = 0;
    if (o.do_combined_histo_pass) {
        combined_histo_elapsed_ms = hist_ms;
        partition_one_elapsed_ms -= hist_ms;
    }
    // (a one-pass plan's empty pass-two stages hold only the events' own gap)
    const float partition_two_elapsed_ms = plan.passes == 2 ? ms[PJ_STAGE_BUILD_PASS2] + ms[PJ_STAGE_PROBE_PASS2] : 0.0f;
    const float data_skew_handle_elapsed_ms = ms[PJ_STAGE_JOIN_PLAN];
    const float join_elapsed_ms = ms[PJ_STAGE_JOIN];
    const float total_elapsed_ms = ms[PJ_STAGE_TOTAL];

    long long num_errors = -1;
    if (!o.skip_cpu_run) {
        unsigned long long* bad_d = nullptr;
        CLI_CUDA(cudaMalloc(&bad_d, sizeof(unsigned long long)));
        CLI_CUDA(cudaMemset(bad_d, 0, sizeof(unsigned long long)));
        const int64_t n = std::min(count, joined_size);
        if (n > 0) verify_pairs_kernel<K><<<1024, 256>>>(br, pr, n, build, nb, probe, np, bad_d);
        CLI_CUDA(cudaGetLastError());
        unsigned long long bad = 0;
        CLI_CUDA(cudaMemcpy(&bad, bad_d, sizeof(bad), cudaMemcpyDeviceToHost));
        CLI_CUDA(cudaFree(bad_d));
        const bool exact = o.uniq_build_tbl_keys && !o.read_from_file && hits >= 0;
        num_errors = static_cast<long long>(bad) + std::llabs(static_cast<long long>(count - joined_size)) +
                     (exact ? std::llabs(static_cast<long long>(count - hits)) : 0);
        if (o.with_value && n > 0) {  // value columns are the row ids: they must equal the rows
            std::vector<int32_t> a(n), b(n), c(n), e(n);
            CLI_CUDA(cudaMemcpy(a.data(), br, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            CLI_CUDA(cudaMemcpy(b.data(), bvo, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            CLI_CUDA(cudaMemcpy(c.data(), pr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            CLI_CUDA(cudaMemcpy(e.data(), pvo, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < n; ++i) num_errors += (a[i] != b[i]) + (c[i] != e[i]);
        }
    }

    if (o.csv) {
        std::cout << count << "," << combined_histo_elapsed_ms << "," << partition_one_elapsed_ms << ","
                  << partition_two_elapsed_ms << "," << data_skew_handle_elapsed_ms << "," << join_elapsed_ms << ","
                  << total_elapsed_ms << "," << num_errors << std::endl;
    } else {
        std::cout << "[*] Results:" << std::endl;
        std::cout << "    joined size          = " << count << std::endl;
        if (o.do_combined_histo_pass)
            std::cout << "    combined histogram time    = " << std::setprecision(3) << combined_histo_elapsed_ms
                      << " ms" << std::endl;
        std::cout << "    partition P1 time    = " << std::setprecision(3) << partition_one_elapsed_ms << " ms"
                  << std::endl;
        if (plan.passes == 2)
            std::cout << "    partition P2 time    = " << std::setprecision(3) << partition_two_elapsed_ms << " ms"
                      << std::endl;
        std::cout << "    skewed data time     = " << std::setprecision(3) << data_skew_handle_elapsed_ms << " ms"
                  << std::endl;
        std::cout << "    join phase time      = " << std::setprecision(3) << join_elapsed_ms << " ms" << std::endl;
        std::cout << "    total exec time      = " << std::setprecision(3) << total_elapsed_ms << " ms" << std::endl;
        const long long input_size = o.with_value ? (np + nb) * static_cast<long long>(sizeof(K) + sizeof(int32_t))
                                                  : (np + nb) * static_cast<long long>(sizeof(K));
        std::cout << "    effective BW         = " << input_size / (total_elapsed_ms / 1000 * 1e9) << " GB/s"
                  << std::endl;
        std::cout << "    device memory usage  = " << device_memory_used / 1e9 << " GB" << std::endl;
        if (!o.skip_cpu_run) {
            std::cout << "    number of errors     = " << num_errors << std::endl;
        } else {
            std::cout << "    reference CPU time   = SKIPPED" << std::endl;
            std::cout << "    number of errors     = SKIPPED" << std::endl;
        }
        if (dev_status == PJ_ERR_CAPACITY)
            std::cout << "    note                 = output size " << joined_size << " < joined size " << count
                      << std::endl;
    }

    cudaFree(build);
    cudaFree(probe);
    cudaFree(hits_d);
    cudaFree(bval);
    cudaFree(pval);
    cudaFree(ws);
    cudaFree(count_d);
    cudaFree(br);
    cudaFree(pr);
    cudaFree(bvo);
    cudaFree(pvo);
    return num_errors > 0 ? 2 : 0;
}

}  // namespace

int main(int argc, char** argv)
{
    Options o = parse(argc, argv);
    if (o.key_bytes != 4 && o.key_bytes != 8) {
        std::cerr << "Error: -K takes 4 or 8." << std::endl;
        return 1;
    }
    return o.key_bytes == 4 ? run<int32_t>(o) : run<int64_t>(o);
}
