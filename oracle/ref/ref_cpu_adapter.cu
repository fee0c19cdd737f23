// ref_cpu_adapter.cu -- C entry points over the reference's own host code.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline).  Compiled by
// oracle/build_ref.sh against the unmodified reference headers
//   src/hash_functions.cuh   MurmurHash3_32<Key>          (:33-119)
//   src/int_fastdiv.h        int_fastdiv, operator%        (:21-175)
//   src/inner_join_cpu.hpp   inner_join_cpu<K,J>           (:24-107)
// into oracle/_ref/libref_cpu.so.  Nothing here is reference source: it only
// instantiates the reference templates and copies results into flat arrays.
#include <algorithm>  // the reference header uses std::stable_sort without including it
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <vector>

#include "hash_functions.cuh"
#include "int_fastdiv.h"
#include "inner_join_cpu.hpp"

extern "C" {

uint32_t ref_murmur_i32(int32_t k)
{
    MurmurHash3_32<int> h;
    return h(static_cast<int>(k));
}

uint32_t ref_murmur_i64(int64_t k)
{
    MurmurHash3_32<long long> h;
    return h(static_cast<long long>(k));
}

// The slot expression of hash_join_kernels.cuh:100-101 evaluated on the host
// with the reference's int_fastdiv (its host branch of operator/ :108).
int32_t ref_slot(uint32_t h, int32_t table_size)
{
    int_fastdiv d(table_size);
    int t = h % d;
    return t < 0 ? -t : t;
}

// inner_join_cpu on the reference's own code path.  Writes the x field
// (the key) of each emitted record into out_keys (at most `capacity`),
// stores the function's own omp_get_wtime() interval in *seconds and
// returns the number of records.  threads <= 0 keeps OpenMP's default.
int64_t ref_inner_join_cpu_i32(const int32_t* build, int64_t n_build, const int32_t* probe,
                               int64_t n_probe, int unique_keys, int32_t* out_keys,
                               int64_t capacity, double* seconds, int threads)
{
    std::vector<int> b(build, build + n_build), p(probe, probe + n_probe);
    std::vector<int2> joined;
    joined.reserve(static_cast<size_t>(unique_keys ? (n_probe > 0 ? n_probe : 1) : 16));
    double t = inner_join_cpu(b, unique_keys != 0, p, joined, threads);
    if (seconds) *seconds = t;
    int64_t n = static_cast<int64_t>(joined.size());
    for (int64_t i = 0; i < n && i < capacity; ++i) out_keys[i] = joined[i].x;
    return n;
}

int64_t ref_inner_join_cpu_i64(const int64_t* build, int64_t n_build, const int64_t* probe,
                               int64_t n_probe, int unique_keys, int64_t* out_keys,
                               int64_t capacity, double* seconds, int threads)
{
    std::vector<long long> b(build, build + n_build), p(probe, probe + n_probe);
    std::vector<longlong2> joined;
    joined.reserve(static_cast<size_t>(unique_keys ? (n_probe > 0 ? n_probe : 1) : 16));
    double t = inner_join_cpu(b, unique_keys != 0, p, joined, threads);
    if (seconds) *seconds = t;
    int64_t n = static_cast<int64_t>(joined.size());
    for (int64_t i = 0; i < n && i < capacity; ++i) out_keys[i] = joined[i].x;
    return n;
}

int ref_omp_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
