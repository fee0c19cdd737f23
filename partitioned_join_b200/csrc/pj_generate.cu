// pj_generate.cu -- seeded input tables generated on the device.
//
// The reference draws its tables with cuRAND on the GPU
// (generate_input_tables.cuh:35-226): build keys from [0, rand_max] (unique
// ones by drawing from a "lottery" array of all candidates), probe keys
// equal to a random build key with probability `selectivity`, else a random
// candidate.  Its Zipf generator (generate_zipf_input.cuh:21-134) samples
// ranks through a CDF table over a random permutation of the alphabet.
//
// Here every draw is a pure function of (seed, row), so a table of any size
// is generated in one pass with no state and no lottery array:
//   * unique build keys: pi(0 .. n_build-1) for a keyed pseudo-random
//     permutation pi of [0, rand_max] (a 4-round Feistel network on the
//     smallest even-bit power of two covering the domain, with cycle
//     walking: Black and Rogaway, "Ciphers with arbitrary finite domains",
//     CT-RSA 2002), so keys are distinct by construction;
//   * repeated build keys: uniform on [0, rand_max];
//   * probe hits: build[i] for i uniform, or i = rho(rank - 1) for a Zipf
//     rank drawn by rejection-inversion (Hormann and Derflinger, "Rejection-
//     inversion to generate variates from monotone discrete distributions",
//     ACM TOMACS 1996) and rho a second keyed permutation (rank -> row);
//   * probe misses: pi(j) for j uniform in [n_build, rand_max] -- exactly the
//     domain values that are not build keys -- or, when the build side uses
//     the whole domain, a uniform value above rand_max.
// Random numbers: SplitMix64 of (seed, stream, row) (Steele, Lea, Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014).
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/pj.h"

namespace {

__host__ __device__ __forceinline__ uint64_t splitmix(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t draw(uint64_t seed, uint64_t stream, uint64_t row)
{
    return splitmix(splitmix(seed ^ (stream * 0xd1b54a32d192ed03ull)) + row);
}

// uniform double in [0, 1) from the top 53 bits
__device__ __forceinline__ double unit(uint64_t r) { return static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0); }

// Keyed permutation of [0, domain).
struct Perm {
    uint64_t domain;
    int half;           // bits of each Feistel half
    uint64_t mask;      // (1 << half) - 1
    uint64_t key[4];

    __host__ void init(uint64_t dom, uint64_t seed)
    {
        domain = dom;
        int bits = 1;
        while (bits < 64 && (uint64_t(1) << bits) < dom) ++bits;
        if (bits & 1) ++bits;
        half = bits / 2;
        mask = (uint64_t(1) << half) - 1;
        for (int i = 0; i < 4; ++i) key[i] = splitmix(seed + 0x632be59bd9b4e019ull * (i + 1));
    }
    __device__ __forceinline__ uint64_t round(uint64_t v) const
    {
        uint64_t l = v >> half, r = v & mask;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint64_t f = splitmix(r ^ key[i]) & mask;
            const uint64_t nl = r;
            r = l ^ f;
            l = nl;
        }
        return (l << half) | r;
    }
    // cycle walking: apply the permutation of [0, 2^(2 half)) until the value
    // falls inside the domain (it returns to x at the latest, so this ends)
    __device__ __forceinline__ uint64_t operator()(uint64_t x) const
    {
        uint64_t v = round(x);
        while (v >= domain) v = round(v);
        return v;
    }
};

// Zipf(s) over ranks 1..n by rejection-inversion: H is an antiderivative of
// the density x^-s, sampled by inversion and corrected by one acceptance test.
struct Zipf {
    double s, n, h_x1, h_n, cut;

    __host__ __device__ static double helper1(double x)  // log1p(x) / x
    {
        return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
    }
    __host__ __device__ static double helper2(double x)  // expm1(x) / x
    {
        return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
    }
    __host__ __device__ double H(double x) const
    {
        const double lx = log(x);
        return helper2((1.0 - s) * lx) * lx;
    }
    __host__ __device__ double H_inv(double x) const
    {
        double t = x * (1.0 - s);
        if (t < -1.0) t = -1.0;
        return exp(helper1(t) * x);
    }
    __host__ __device__ double h(double x) const { return exp(-s * log(x)); }

    __host__ void init(double exponent, int64_t count)
    {
        s = exponent;
        n = static_cast<double>(count);
        h_x1 = H(1.5) - 1.0;
        h_n = H(n + 0.5);
        cut = 2.0 - H_inv(H(2.5) - h(2.0));
    }
    // rank in [1, n]
    __device__ int64_t sample(uint64_t seed, uint64_t stream, uint64_t row) const
    {
        double k = 1.0;
        for (int attempt = 0; attempt < 64; ++attempt) {
            const double u = h_n + unit(draw(seed, stream + attempt, row)) * (h_x1 - h_n);
            const double x = H_inv(u);
            k = floor(x + 0.5);
            if (k < 1.0) k = 1.0;
            if (k > n) k = n;
            if (k - x <= cut || u >= H(k + 0.5) - h(k)) break;
        }
        return static_cast<int64_t>(k);
    }
};

enum : uint64_t { S_BUILD = 1, S_HIT = 2, S_PICK = 3, S_MISS = 4, S_ZIPF = 16 };

template <typename K>
__global__ void gen_build_kernel(K* __restrict__ out, int64_t n, int64_t rand_max, int32_t unique, Perm pi,
                                 uint64_t seed)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint64_t v;
        if (unique) {
            v = pi(static_cast<uint64_t>(i));
        } else {
            const uint64_t dom = static_cast<uint64_t>(rand_max) + 1;
            v = static_cast<uint64_t>(unit(draw(seed, S_BUILD, i)) * static_cast<double>(dom));
            if (v >= dom) v = dom - 1;
        }
        out[i] = static_cast<K>(v);
    }
}

template <typename K>
__global__ void gen_probe_kernel(K* __restrict__ out, int64_t n, const K* __restrict__ build, int64_t n_build,
                                 int64_t rand_max, int64_t key_max, double selectivity, int32_t unique, Perm pi,
                                 Perm rho, int32_t zipf, Zipf z, uint64_t seed, unsigned long long* hits)
{
    unsigned long long mine = 0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const bool hit = n_build > 0 && unit(draw(seed, S_HIT, i)) < selectivity;
        K v;
        if (hit) {
            int64_t j;
            if (zipf) {
                j = static_cast<int64_t>(rho(static_cast<uint64_t>(z.sample(seed, S_ZIPF, i) - 1)));
            } else {
                j = static_cast<int64_t>(unit(draw(seed, S_PICK, i)) * static_cast<double>(n_build));
                if (j >= n_build) j = n_build - 1;
            }
            v = build[j];
            ++mine;
        } else {
            const uint64_t dom = static_cast<uint64_t>(rand_max) + 1;
            const double u = unit(draw(seed, S_MISS, i));
            if (unique && dom > static_cast<uint64_t>(n_build)) {
                // a domain value that no build row drew
                uint64_t j = static_cast<uint64_t>(n_build) +
                             static_cast<uint64_t>(u * static_cast<double>(dom - static_cast<uint64_t>(n_build)));
                if (j >= dom) j = dom - 1;
                v = static_cast<K>(pi(j));
            } else {
                // above the domain
                const double span = static_cast<double>(key_max) - static_cast<double>(rand_max);
                int64_t x = rand_max + 1 + static_cast<int64_t>(u * (span > 1.0 ? span - 1.0 : 0.0));
                if (x > key_max) x = key_max;
                v = static_cast<K>(x);
            }
        }
        out[i] = v;
    }
    if (hits) {
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(hits, mine);
    }
}

unsigned grid_of(int64_t n)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    const int64_t g = (n + 255) / 256;
    const int64_t cap = static_cast<int64_t>(sms) * 16;
    return static_cast<unsigned>(g < 1 ? 1 : (g < cap ? g : cap));
}

template <typename K>
pj_status generate(K* build, int64_t n_build, K* probe, int64_t n_probe, int64_t rand_max, double selectivity,
                   int32_t unique, double zipf_theta, uint64_t seed, int64_t* hits, cudaStream_t st)
{
    const int64_t key_max = sizeof(K) == 4 ? INT32_MAX : INT64_MAX;
    if (rand_max < 0 || rand_max >= key_max) return PJ_ERR_INVALID;
    if (unique && static_cast<uint64_t>(rand_max) + 1 < static_cast<uint64_t>(n_build)) return PJ_ERR_INVALID;
    Perm pi, rho;
    pi.init(static_cast<uint64_t>(rand_max) + 1, seed ^ 0x5851f42d4c957f2dull);
    rho.init(n_build > 0 ? static_cast<uint64_t>(n_build) : 1, seed ^ 0x14057b7ef767814full);
    Zipf z{};
    const int32_t zipf = zipf_theta > 0.0 ? 1 : 0;
    if (zipf) z.init(zipf_theta, n_build > 0 ? n_build : 1);
    if (hits && cudaMemsetAsync(hits, 0, sizeof(int64_t), st) != cudaSuccess) return PJ_ERR_CUDA;
    if (n_build > 0) gen_build_kernel<K><<<grid_of(n_build), 256, 0, st>>>(build, n_build, rand_max, unique, pi, seed);
    if (n_probe > 0)
        gen_probe_kernel<K><<<grid_of(n_probe), 256, 0, st>>>(probe, n_probe, build, n_build, rand_max, key_max,
                                                              selectivity, unique, pi, rho, zipf, z, seed,
                                                              reinterpret_cast<unsigned long long*>(hits));
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

}  // namespace

extern "C" pj_status pj_generate_tables(void* build_keys, int64_t n_build, void* probe_keys, int64_t n_probe,
                                        int32_t key_bytes, int64_t rand_max, double selectivity,
                                        int32_t unique_build_keys, double zipf_theta, uint64_t seed,
                                        int64_t* hits_dev, pj_stream stream)
{
    if (n_build < 0 || n_probe < 0 || (n_build > 0 && !build_keys) || (n_probe > 0 && !probe_keys)) return PJ_ERR_INVALID;
    if (key_bytes != 4 && key_bytes != 8) return PJ_ERR_INVALID;
    if (!(selectivity >= 0.0 && selectivity <= 1.0) || !(zipf_theta >= 0.0 && zipf_theta <= 10.0)) return PJ_ERR_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (key_bytes == 4)
        return generate<int32_t>(static_cast<int32_t*>(build_keys), n_build, static_cast<int32_t*>(probe_keys), n_probe,
                                 rand_max, selectivity, unique_build_keys, zipf_theta, seed, hits_dev, st);
    return generate<int64_t>(static_cast<int64_t*>(build_keys), n_build, static_cast<int64_t*>(probe_keys), n_probe,
                             rand_max, selectivity, unique_build_keys, zipf_theta, seed, hits_dev, st);
}
