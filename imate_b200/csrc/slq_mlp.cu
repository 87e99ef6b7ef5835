// Learned surrogate of a parameter sweep t -> trace f(A + t I).
//
// imate interpolates such sweeps from a few exact or SLQ evaluations
// (imate/interpolator/, InterpolateSchatten interpolate_schatten.py:426-492).
// Here a small fully connected network 1 -> 64 -> 64 -> 1 (tanh hidden
// units, FP32) is fitted on the device to SLQ samples of the sweep and then
// answers the whole sweep in one launch.  Training is full-batch Adam on the
// mean squared error, all steps inside one CTA (the batch is a few dozen
// points, the network 4353 parameters), so a fit is a single launch.
//
// Parameter layout (float, P = 4353):
//   W1[64] | b1[64] | W2[64][64] (row k = weights into unit k) | b2[64] |
//   W3[64] | b3[1]

#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/slq.h"

namespace {

constexpr int H = SLQ_MLP_WIDTH;
constexpr int P = SLQ_MLP_PARAMS;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int MAX_BATCH = SLQ_MLP_MAX_BATCH;

}  // namespace

namespace slq {
void set_error(const std::string& message);  // slq_engine.cu
}

namespace {

slq_status mlp_fail(slq_status s, const std::string& m)
{
    slq::set_error(m);
    return s;
}

// Forward pass of one input, parameters in shared memory.
__device__ float mlp_eval(const float* p, float x)
{
    float h1[H];
#pragma unroll 8
    for (int j = 0; j < H; ++j) h1[j] = tanhf(p[OFF_W1 + j] * x + p[OFF_B1 + j]);
    float y = p[OFF_B3];
    for (int k = 0; k < H; ++k)
    {
        float z = p[OFF_B2 + k];
        const float* w = p + OFF_W2 + k * H;
#pragma unroll 8
        for (int j = 0; j < H; ++j) z += w[j] * h1[j];
        y += p[OFF_W3 + k] * tanhf(z);
    }
    return y;
}

__global__ void k_mlp_forward(const float* __restrict__ params, const float* __restrict__ x,
                              int count, float* __restrict__ y)
{
    __shared__ float p[P];
    for (int i = threadIdx.x; i < P; i += blockDim.x) p[i] = params[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) y[i] = mlp_eval(p, x[i]);
}

// Shared state of one training step over a batch of B <= MAX_BATCH points.
struct StepSmem {
    float p[P];
    float g[P];
    float h1[MAX_BATCH][H];
    float h2[MAX_BATCH][H];
    float dz2[MAX_BATCH][H];
    float dz1[MAX_BATCH][H];
    float dy[MAX_BATCH];
    float loss;
};

// Gradient of L = mean_i (y_i - t_i)^2 into s.g (and the loss).
__device__ void mlp_grad_block(StepSmem& s, const float* x, const float* t, int B)
{
    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    // layer 1
    for (int e = tid; e < B * H; e += nt)
    {
        const int i = e / H, j = e % H;
        s.h1[i][j] = tanhf(s.p[OFF_W1 + j] * x[i] + s.p[OFF_B1 + j]);
    }
    __syncthreads();
    // layer 2
    for (int e = tid; e < B * H; e += nt)
    {
        const int i = e / H, k = e % H;
        float z = s.p[OFF_B2 + k];
        const float* w = s.p + OFF_W2 + k * H;
        for (int j = 0; j < H; ++j) z += w[j] * s.h1[i][j];
        s.h2[i][k] = tanhf(z);
    }
    __syncthreads();
    // output and dL/dy (one warp per point)
    const int lane = tid & 31;
    for (int i = tid >> 5; i < B; i += nt >> 5)
    {
        float y = 0.0f;
        for (int k = lane; k < H; k += 32) y += s.p[OFF_W3 + k] * s.h2[i][k];
        for (int off = 16; off > 0; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
        if (lane == 0)
        {
            y += s.p[OFF_B3];
            s.dy[i] = 2.0f * (y - t[i]) / B;
        }
    }
    __syncthreads();
    if (tid == 0)
    {
        float l = 0.0f;
        for (int i = 0; i < B; ++i)
        {
            const float r = s.dy[i] * B * 0.5f;
            l += r * r;
        }
        s.loss = l / B;
    }
    // dz2 = dy * W3 * (1 - h2^2)
    for (int e = tid; e < B * H; e += nt)
    {
        const int i = e / H, k = e % H;
        const float h = s.h2[i][k];
        s.dz2[i][k] = s.dy[i] * s.p[OFF_W3 + k] * (1.0f - h * h);
    }
    __syncthreads();
    // dz1 = (W2^T dz2) * (1 - h1^2)
    for (int e = tid; e < B * H; e += nt)
    {
        const int i = e / H, j = e % H;
        float d = 0.0f;
        for (int k = 0; k < H; ++k) d += s.p[OFF_W2 + k * H + j] * s.dz2[i][k];
        const float h = s.h1[i][j];
        s.dz1[i][j] = d * (1.0f - h * h);
    }
    __syncthreads();
    // parameter gradients
    for (int q = tid; q < P; q += nt)
    {
        float gsum = 0.0f;
        if (q < OFF_B1)
        {
            for (int i = 0; i < B; ++i) gsum += s.dz1[i][q] * x[i];
        }
        else if (q < OFF_W2)
        {
            const int j = q - OFF_B1;
            for (int i = 0; i < B; ++i) gsum += s.dz1[i][j];
        }
        else if (q < OFF_B2)
        {
            const int k = (q - OFF_W2) / H, j = (q - OFF_W2) % H;
            for (int i = 0; i < B; ++i) gsum += s.dz2[i][k] * s.h1[i][j];
        }
        else if (q < OFF_W3)
        {
            const int k = q - OFF_B2;
            for (int i = 0; i < B; ++i) gsum += s.dz2[i][k];
        }
        else if (q < OFF_B3)
        {
            const int k = q - OFF_W3;
            for (int i = 0; i < B; ++i) gsum += s.dy[i] * s.h2[i][k];
        }
        else
        {
            for (int i = 0; i < B; ++i) gsum += s.dy[i];
        }
        s.g[q] = gsum;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(512)
k_mlp_grad(const float* __restrict__ params, const float* __restrict__ x,
           const float* __restrict__ t, int B, float* __restrict__ grad,
           float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_mlp[];
    StepSmem& s = *reinterpret_cast<StepSmem*>(smem_mlp);
    __shared__ float xs[MAX_BATCH], ts[MAX_BATCH];
    for (int i = threadIdx.x; i < P; i += blockDim.x) s.p[i] = params[i];
    for (int i = threadIdx.x; i < B; i += blockDim.x)
    {
        xs[i] = x[i];
        ts[i] = t[i];
    }
    __syncthreads();
    mlp_grad_block(s, xs, ts, B);
    for (int i = threadIdx.x; i < P; i += blockDim.x) grad[i] = s.g[i];
    if (threadIdx.x == 0) *loss = s.loss;
}

// Full-batch Adam (Kingma & Ba), `steps` iterations in one CTA.  m, v are
// the first/second moment estimates (device, P each) and persist across
// calls; step0 is the number of steps already taken (bias correction).
__global__ void __launch_bounds__(512)
k_mlp_train(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
            const float* __restrict__ x, const float* __restrict__ t, int B, int steps,
            int step0, float lr, float beta1, float beta2, float eps,
            float* __restrict__ loss_out)
{
    extern __shared__ __align__(16) unsigned char smem_mlp[];
    StepSmem& s = *reinterpret_cast<StepSmem*>(smem_mlp);
    __shared__ float xs[MAX_BATCH], ts[MAX_BATCH];
    for (int i = threadIdx.x; i < P; i += blockDim.x) s.p[i] = params[i];
    for (int i = threadIdx.x; i < B; i += blockDim.x)
    {
        xs[i] = x[i];
        ts[i] = t[i];
    }
    __syncthreads();
    float b1t = powf(beta1, static_cast<float>(step0));
    float b2t = powf(beta2, static_cast<float>(step0));
    for (int it = 0; it < steps; ++it)
    {
        mlp_grad_block(s, xs, ts, B);
        b1t *= beta1;
        b2t *= beta2;
        const float c1 = 1.0f / (1.0f - b1t);
        const float c2 = 1.0f / (1.0f - b2t);
        for (int q = threadIdx.x; q < P; q += blockDim.x)
        {
            const float g = s.g[q];
            const float mq = beta1 * m[q] + (1.0f - beta1) * g;
            const float vq = beta2 * v[q] + (1.0f - beta2) * g * g;
            m[q] = mq;
            v[q] = vq;
            s.p[q] -= lr * (mq * c1) / (sqrtf(vq * c2) + eps);
        }
        if (threadIdx.x == 0 && loss_out) loss_out[it] = s.loss;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) params[i] = s.p[i];
}

size_t step_smem() { return sizeof(StepSmem); }

slq_status set_smem_attr()
{
    static bool done = false;
    if (done) return SLQ_OK;
    const int bytes = static_cast<int>(step_smem());
    cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess)
        return mlp_fail(SLQ_ERR_CUDA, std::string("mlp smem attribute: ") + cudaGetErrorString(e));
    done = true;
    return SLQ_OK;
}

}  // namespace

extern "C" slq_status slq_mlp_forward(const float* params, const float* x, int count, float* y,
                                      void* stream)
{
    if (!params || !x || !y || count < 0) return mlp_fail(SLQ_ERR_BAD_ARG, "mlp_forward: bad argument");
    if (count == 0) return SLQ_OK;
    k_mlp_forward<<<(count + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(params, x,
                                                                                     count, y);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mlp_fail(SLQ_ERR_CUDA, cudaGetErrorString(e));
    return SLQ_OK;
}

extern "C" slq_status slq_mlp_grad(const float* params, const float* x, const float* t,
                                   int batch, float* grad, float* loss, void* stream)
{
    if (!params || !x || !t || !grad || !loss || batch < 1 || batch > MAX_BATCH)
        return mlp_fail(SLQ_ERR_BAD_ARG, "mlp_grad: bad argument (batch <= " +
                                             std::to_string(MAX_BATCH) + ")");
    slq_status st = set_smem_attr();
    if (st != SLQ_OK) return st;
    k_mlp_grad<<<1, 512, step_smem(), static_cast<cudaStream_t>(stream)>>>(params, x, t, batch,
                                                                          grad, loss);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mlp_fail(SLQ_ERR_CUDA, cudaGetErrorString(e));
    return SLQ_OK;
}

extern "C" slq_status slq_mlp_train(float* params, float* adam_m, float* adam_v, const float* x,
                                    const float* t, int batch, int steps, int steps_done,
                                    float lr, float* loss_history, void* stream)
{
    if (!params || !adam_m || !adam_v || !x || !t || batch < 1 || batch > MAX_BATCH ||
        steps < 0 || steps_done < 0 || !(lr > 0.0f))
        return mlp_fail(SLQ_ERR_BAD_ARG, "mlp_train: bad argument");
    slq_status st = set_smem_attr();
    if (st != SLQ_OK) return st;
    k_mlp_train<<<1, 512, step_smem(), static_cast<cudaStream_t>(stream)>>>(
        params, adam_m, adam_v, x, t, batch, steps, steps_done, lr, 0.9f, 0.999f, 1e-8f,
        loss_history);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mlp_fail(SLQ_ERR_CUDA, cudaGetErrorString(e));
    return SLQ_OK;
}
