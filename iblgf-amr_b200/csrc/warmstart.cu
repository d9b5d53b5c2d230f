// Learned warm start of the immersed-boundary force CG: a small 1-D
// convolutional network over the IB points, FP32,
// with hand-written forward, backward and Adam kernels.
//
//   x  [S][9][N]   inputs, points in Morton order of their coordinates: the
//                  change of the CG right-hand side (velocity at the points)
//                  since the previous step (3), the stage's previous force (3)
//                  and its last change f_prev - f_prev2 (3), each scaled by a
//                  fixed rms. The Schur operator A is constant in time, so the
//                  target f - f_prev = A^-1 (uc - uc_prev); the last force
//                  change gives the network the extrapolation in time
//   h1 = relu(conv5(x;  W1 [64][9][5],  b1))      [S][64][N]
//   h2 = relu(conv5(h1; W2 [64][64][5], b2))      [S][64][N]
//   y  =      conv5(h2; W3 [3][64][5],  b3)       [S][3][N]
// conv5: kernel 5, zero padding 2, stride 1 (24 451 parameters). The warm
// start is f0 = f_prev + s_t * y, s_t the rms of f - f_prev in the samples;
// the CG then runs to its unchanged tolerance. Loss: mean squared error
// against (f - f_prev) / s_t over the samples.
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
constexpr int kK = 5, kPad = 2;

// y[s][co][n] = b[co] + sum_ci sum_k W[co][ci][k] x[s][ci][n + k - 2]
__global__ void conv_fwd_kernel(const float* __restrict__ x, const float* __restrict__ W, const float* __restrict__ b,
                                float* __restrict__ y, int S, int ci_n, int co_n, int N, int relu)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)S * co_n * N) return;
    const int n = (int)(t % N), co = (int)((t / N) % co_n), s = (int)(t / ((long long)N * co_n));
    float acc = b[co];
    const float* xs = x + (size_t)s * ci_n * N;
    const float* w = W + (size_t)co * ci_n * kK;
    for (int ci = 0; ci < ci_n; ++ci)
#pragma unroll
        for (int k = 0; k < kK; ++k)
        {
            const int m = n + k - kPad;
            if (m >= 0 && m < N) acc = fmaf(w[ci * kK + k], xs[(size_t)ci * N + m], acc);
        }
    y[t] = relu ? fmaxf(acc, 0.0f) : acc;
}

// dx[s][ci][n] = (sum_co sum_k W[co][ci][k] dy[s][co][n - k + 2]) * (h > 0 if masked)
__global__ void conv_bwd_input_kernel(const float* __restrict__ dy, const float* __restrict__ W,
                                      const float* __restrict__ h, float* __restrict__ dx, int S, int ci_n, int co_n,
                                      int N)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)S * ci_n * N) return;
    const int n = (int)(t % N), ci = (int)((t / N) % ci_n), s = (int)(t / ((long long)N * ci_n));
    float acc = 0.0f;
    const float* dys = dy + (size_t)s * co_n * N;
    for (int co = 0; co < co_n; ++co)
#pragma unroll
        for (int k = 0; k < kK; ++k)
        {
            const int m = n - k + kPad;
            if (m >= 0 && m < N) acc = fmaf(W[((size_t)co * ci_n + ci) * kK + k], dys[(size_t)co * N + m], acc);
        }
    if (h && h[t] <= 0.0f) acc = 0.0f;
    dx[t] = acc;
}

// one CTA per weight (co, ci, k) or bias (ci = -1): block reduction over (s, n)
__global__ void conv_bwd_weight_kernel(const float* __restrict__ dy, const float* __restrict__ x,
                                       float* __restrict__ dW, float* __restrict__ db, int S, int ci_n, int co_n,
                                       int N)
{
    const int wid = blockIdx.x;
    const int nw = co_n * ci_n * kK;
    const bool bias = wid >= nw;
    const int co = bias ? wid - nw : wid / (ci_n * kK);
    const int ci = bias ? 0 : (wid / kK) % ci_n, k = bias ? 0 : wid % kK;
    float acc = 0.0f;
    for (long long i = threadIdx.x; i < (long long)S * N; i += blockDim.x)
    {
        const int s = (int)(i / N), n = (int)(i % N);
        const float g = dy[((size_t)s * co_n + co) * N + n];
        if (bias) acc += g;
        else
        {
            const int m = n + k - kPad;
            if (m >= 0 && m < N) acc = fmaf(g, x[((size_t)s * ci_n + ci) * N + m], acc);
        }
    }
    __shared__ float red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        if (bias) db[co] = red[0];
        else dW[wid] = red[0];
    }
}

// dy = 2 (y - t) / count; loss accumulated per CTA then summed on the host
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ tgt, float* __restrict__ dy,
                                long long count, float* __restrict__ partial)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < count)
    {
        const float d = y[i] - tgt[i];
        dy[i] = 2.0f * d / (float)count;
        l = d * d / (float)count;
    }
    __shared__ float red[256];
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }
}  // namespace

// parameter layout: W1 b1 W2 b2 W3 b3
void ws_offsets(int* off)
{
    const int C = kWsChannels;
    off[0] = 0;
    off[1] = off[0] + C * kWsInputs * kK;
    off[2] = off[1] + C;
    off[3] = off[2] + C * C * kK;
    off[4] = off[3] + C;
    off[5] = off[4] + 3 * C * kK;
    off[6] = off[5] + 3;
}

void ws_forward(Ctx& c, const float* params, const float* x, int S, int N, float* h1, float* h2, float* y)
{
    int o[7];
    ws_offsets(o);
    const int C = kWsChannels;
    conv_fwd_kernel<<<blocks_for((long long)S * C * N, 128), 128, 0, c.stream>>>(x, params + o[0], params + o[1], h1,
                                                                               S, kWsInputs, C, N, 1);
    conv_fwd_kernel<<<blocks_for((long long)S * C * N, 128), 128, 0, c.stream>>>(h1, params + o[2], params + o[3],
                                                                               h2, S, C, C, N, 1);
    conv_fwd_kernel<<<blocks_for((long long)S * 3 * N, 128), 128, 0, c.stream>>>(h2, params + o[4], params + o[5], y,
                                                                               S, C, 3, N, 0);
    c.launches += 3;
    IBLGF_CUDA(cudaGetLastError());
}

// gradients of the mean squared error; returns the loss (host synchronises)
float ws_backward(Ctx& c, const float* params, const float* x, const float* tgt, int S, int N, const float* h1,
                  const float* h2, const float* y, float* dy, float* dh2, float* dh1, float* grads,
                  DevBuf<float>& partial)
{
    int o[7];
    ws_offsets(o);
    const int C = kWsChannels;
    const long long cnt = (long long)S * 3 * N;
    const unsigned nb = blocks_for(cnt, 256);
    if (partial.n < nb) partial.alloc(nb);
    mse_grad_kernel<<<nb, 256, 0, c.stream>>>(y, tgt, dy, cnt, partial.p);
    conv_bwd_weight_kernel<<<3 * C * kK + 3, 256, 0, c.stream>>>(dy, h2, grads + o[4], grads + o[5], S, C, 3, N);
    conv_bwd_input_kernel<<<blocks_for((long long)S * C * N, 128), 128, 0, c.stream>>>(dy, params + o[4], h2, dh2, S,
                                                                                     C, 3, N);
    conv_bwd_weight_kernel<<<C * C * kK + C, 256, 0, c.stream>>>(dh2, h1, grads + o[2], grads + o[3], S, C, C, N);
    conv_bwd_input_kernel<<<blocks_for((long long)S * C * N, 128), 128, 0, c.stream>>>(dh2, params + o[2], h1, dh1, S,
                                                                                     C, C, N);
    conv_bwd_weight_kernel<<<C * kWsInputs * kK + C, 256, 0, c.stream>>>(dh1, x, grads + o[0], grads + o[1], S,
                                                                         kWsInputs, C, N);
    c.launches += 6;
    IBLGF_CUDA(cudaGetLastError());
    std::vector<float> h(nb);
    IBLGF_CUDA(cudaMemcpyAsync(h.data(), partial.p, nb * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    double l = 0.0;
    for (float v : h) l += v;
    return (float)l;
}

void ws_adam(Ctx& c, float* params, const float* grads, float* m, float* v, int n, float lr, int step)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    adam_kernel<<<blocks_for(n, 256), 256, 0, c.stream>>>(params, grads, m, v, n, lr, b1, b2, 1e-8f, c1, c2);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
