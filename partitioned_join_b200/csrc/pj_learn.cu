// pj_learn.cu -- the learned planner's network: a two-hidden-layer MLP in
// FP32 with hand-written forward, backward and Adam kernels, and the
// feature sketch it reads.
//
// No reference counterpart: the reference's schedule is fixed by its -n/-N/-f
// flags (main.cu:100-188).  The planner (pj_plan_learned in pj_api.cu) uses
// the network to rank candidate schedules; the join's own device checks
// (table overflow) send a bad choice back to the exact planner, so the
// network can change the schedule but never the result.
//
// Layout of the parameter vector (row-major, ReLU after both hidden layers):
//   W1[in][h1], b1[h1], W2[h1][h2], b2[h2], W3[h2][out], b3[out]
// Saved activations of a forward pass (for backward), per sample row:
//   Z1[h1], A1[h1], Z2[h2], A2[h2]
// The kernels are plain SIMT loops: the network has ~7 K weights and the
// batches a few thousand rows, far from any tensor-core shape.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/pj.h"
#include "pj_device.cuh"

namespace {

struct Dims {
    int in, h1, h2, out;
    __host__ __device__ int64_t w1() const { return 0; }
    __host__ __device__ int64_t b1() const { return static_cast<int64_t>(in) * h1; }
    __host__ __device__ int64_t w2() const { return b1() + h1; }
    __host__ __device__ int64_t b2() const { return w2() + static_cast<int64_t>(h1) * h2; }
    __host__ __device__ int64_t w3() const { return b2() + h2; }
    __host__ __device__ int64_t b3() const { return w3() + static_cast<int64_t>(h2) * out; }
    __host__ __device__ int64_t total() const { return b3() + out; }
    __host__ __device__ int act_stride() const { return 2 * h1 + 2 * h2; }
};

Dims dims_of(const pj_mlp_dims* d) { return Dims{d->in, d->h1, d->h2, d->out}; }

bool valid(const pj_mlp_dims* d)
{
    return d && d->in > 0 && d->h1 > 0 && d->h2 > 0 && d->out > 0 && d->in <= 4096 && d->h1 <= 1024 &&
           d->h2 <= 1024 && d->out <= 1024;
}

unsigned grid_for(int64_t n) { return static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 65535)); }

// Y[b][j] = act(sum_i X[b][i] W[i][j] + bias[j]); also stores Z (pre-activation).
__global__ void dense_forward_kernel(const float* __restrict__ X, int ldx, const float* __restrict__ W,
                                     const float* __restrict__ bias, int in, int out, int batch, int relu,
                                     float* __restrict__ Z, float* __restrict__ Y, int ldy)
{
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < static_cast<int64_t>(batch) * out;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(t / out), j = static_cast<int>(t % out);
        float acc = bias[j];
        const float* x = X + static_cast<int64_t>(b) * ldx;
        for (int i = 0; i < in; ++i) acc = fmaf(x[i], W[static_cast<int64_t>(i) * out + j], acc);
        if (Z) Z[static_cast<int64_t>(b) * ldy + j] = acc;
        Y[static_cast<int64_t>(b) * ldy + j] = relu ? fmaxf(acc, 0.0f) : acc;
    }
}

// dZ = dA * (Z > 0), in place on dA (ReLU backward)
__global__ void relu_backward_kernel(float* __restrict__ dA, const float* __restrict__ Z, int ldz, int width, int batch,
                                     int ldd)
{
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < static_cast<int64_t>(batch) * width;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(t / width), j = static_cast<int>(t % width);
        if (Z[static_cast<int64_t>(b) * ldz + j] <= 0.0f) dA[static_cast<int64_t>(b) * ldd + j] = 0.0f;
    }
}

// dW[i][j] = sum_b X[b][i] dZ[b][j]; db[j] = sum_b dZ[b][j]
__global__ void dense_weight_grad_kernel(const float* __restrict__ X, int ldx, const float* __restrict__ dZ, int ldd,
                                         int in, int out, int batch, float* __restrict__ dW, float* __restrict__ db)
{
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < static_cast<int64_t>(in + 1) * out;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(t / out), j = static_cast<int>(t % out);
        float acc = 0.0f;
        if (i < in) {
            for (int b = 0; b < batch; ++b)
                acc = fmaf(X[static_cast<int64_t>(b) * ldx + i], dZ[static_cast<int64_t>(b) * ldd + j], acc);
            dW[static_cast<int64_t>(i) * out + j] = acc;
        } else {
            for (int b = 0; b < batch; ++b) acc += dZ[static_cast<int64_t>(b) * ldd + j];
            db[j] = acc;
        }
    }
}

// dX[b][i] = sum_j dZ[b][j] W[i][j]
__global__ void dense_input_grad_kernel(const float* __restrict__ dZ, int ldd, const float* __restrict__ W, int in,
                                        int out, int batch, float* __restrict__ dX, int ldx)
{
    for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < static_cast<int64_t>(batch) * in;
         t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(t / in), i = static_cast<int>(t % in);
        float acc = 0.0f;
        const float* dz = dZ + static_cast<int64_t>(b) * ldd;
        const float* w = W + static_cast<int64_t>(i) * out;
        for (int j = 0; j < out; ++j) acc = fmaf(dz[j], w[j], acc);
        dX[static_cast<int64_t>(b) * ldx + i] = acc;
    }
}

// Masked mean squared error: dy = 2 (y - t) m / sum(m); loss = sum m (y - t)^2 / sum(m)
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ target,
                                const float* __restrict__ mask, int64_t n, float* __restrict__ dy, float* loss)
{
    __shared__ float s_sum[2];
    if (threadIdx.x < 2) s_sum[threadIdx.x] = 0.0f;
    __syncthreads();
    float msum = 0.0f, lsum = 0.0f;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float m = mask ? mask[i] : 1.0f;
        const float d = y[i] - target[i];
        msum += m;
        lsum += m * d * d;
    }
    atomicAdd(&s_sum[0], msum);
    atomicAdd(&s_sum[1], lsum);
    __syncthreads();
    const float denom = fmaxf(s_sum[0], 1.0f);
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float m = mask ? mask[i] : 1.0f;
        dy[i] = 2.0f * (y[i] - target[i]) * m / denom;
    }
    if (threadIdx.x == 0 && loss) *loss = s_sum[1] / denom;
}

// Adam (Kingma and Ba, 2015) with bias correction.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace

extern "C" {

int64_t pj_mlp_param_count(const pj_mlp_dims* d) { return valid(d) ? dims_of(d).total() : -1; }

pj_status pj_mlp_forward(const float* params, const pj_mlp_dims* d, const float* x, int32_t batch, float* acts,
                         float* y, pj_stream stream)
{
    if (!valid(d) || !params || batch < 0 || (batch > 0 && (!x || !y))) return PJ_ERR_INVALID;
    if (batch == 0) return PJ_OK;
    const Dims D = dims_of(d);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int S = D.act_stride();
    if (!acts) return PJ_ERR_INVALID;  // hidden activations: batch x act_stride floats
    float* Z1 = acts;
    float* A1 = acts + D.h1;
    float* Z2 = acts + 2 * D.h1;
    float* A2 = acts + 2 * D.h1 + D.h2;
    dense_forward_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h1), 256, 0, st>>>(
        x, D.in, params + D.w1(), params + D.b1(), D.in, D.h1, batch, 1, Z1, A1, S);
    dense_forward_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h2), 256, 0, st>>>(
        A1, S, params + D.w2(), params + D.b2(), D.h1, D.h2, batch, 1, Z2, A2, S);
    dense_forward_kernel<<<grid_for(static_cast<int64_t>(batch) * D.out), 256, 0, st>>>(
        A2, S, params + D.w3(), params + D.b3(), D.h2, D.out, batch, 0, nullptr, y, D.out);
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

pj_status pj_mlp_backward(const float* params, const pj_mlp_dims* d, const float* x, const float* acts,
                          const float* dy, int32_t batch, float* grad, float* scratch, pj_stream stream)
{
    if (!valid(d) || !params || !acts || !dy || !grad || !scratch || batch <= 0 || !x) return PJ_ERR_INVALID;
    const Dims D = dims_of(d);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int S = D.act_stride();
    const float* Z1 = acts;
    const float* A1 = acts + D.h1;
    const float* Z2 = acts + 2 * D.h1;
    const float* A2 = acts + 2 * D.h1 + D.h2;
    float* dA2 = scratch;                                   // batch x h2
    float* dA1 = scratch + static_cast<int64_t>(batch) * D.h2;  // batch x h1
    // layer 3
    dense_weight_grad_kernel<<<grid_for(static_cast<int64_t>(D.h2 + 1) * D.out), 256, 0, st>>>(
        A2, S, dy, D.out, D.h2, D.out, batch, grad + D.w3(), grad + D.b3());
    dense_input_grad_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h2), 256, 0, st>>>(
        dy, D.out, params + D.w3(), D.h2, D.out, batch, dA2, D.h2);
    relu_backward_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h2), 256, 0, st>>>(dA2, Z2, S, D.h2, batch, D.h2);
    // layer 2
    dense_weight_grad_kernel<<<grid_for(static_cast<int64_t>(D.h1 + 1) * D.h2), 256, 0, st>>>(
        A1, S, dA2, D.h2, D.h1, D.h2, batch, grad + D.w2(), grad + D.b2());
    dense_input_grad_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h1), 256, 0, st>>>(
        dA2, D.h2, params + D.w2(), D.h1, D.h2, batch, dA1, D.h1);
    relu_backward_kernel<<<grid_for(static_cast<int64_t>(batch) * D.h1), 256, 0, st>>>(dA1, Z1, S, D.h1, batch, D.h1);
    // layer 1
    dense_weight_grad_kernel<<<grid_for(static_cast<int64_t>(D.in + 1) * D.h1), 256, 0, st>>>(
        x, D.in, dA1, D.h1, D.in, D.h1, batch, grad + D.w1(), grad + D.b1());
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

pj_status pj_mlp_mse_grad(const float* y, const float* target, const float* mask, int64_t n, float* dy, float* loss,
                          pj_stream stream)
{
    if (!y || !target || !dy || n < 0) return PJ_ERR_INVALID;
    if (n == 0) return PJ_OK;
    mse_grad_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(y, target, mask, n, dy, loss);
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

pj_status pj_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t n, float lr, float beta1,
                      float beta2, float eps, int32_t step, pj_stream stream)
{
    if (!params || !grad || !m || !v || n < 0 || step < 1) return PJ_ERR_INVALID;
    const float c1 = 1.0f - powf(beta1, static_cast<float>(step));
    const float c2 = 1.0f - powf(beta2, static_cast<float>(step));
    adam_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grad, m, v, n, lr, beta1, beta2, eps,
                                                                            c1, c2);
    return cudaGetLastError() == cudaSuccess ? PJ_OK : PJ_ERR_CUDA;
}

}  // extern "C"
