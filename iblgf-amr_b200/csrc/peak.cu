// FMA-throughput probe: the FP64 / FP32 CUDA-core roofline denominator that
// the driver-measured peaks (HBM copy, bf16 GEMM) do not cover. Each thread
// runs 8 independent register-resident FMA chains; grid = 8 CTAs per SM.
#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
template<class R>
__global__ void __launch_bounds__(256) fma_chain_kernel(R* out, int iters, R a, R b)
{
    R x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (R)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    R s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == (R)-1.2345) out[0] = s;  // keeps the chains live
}

template<class R>
double run(Ctx& c)
{
    int dev = 0, sms = 0;
    IBLGF_CUDA(cudaGetDevice(&dev));
    IBLGF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DevBuf<R> out;
    out.alloc(1);
    const int iters = 1 << 14, blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    IBLGF_CUDA(cudaEventCreate(&e0));
    IBLGF_CUDA(cudaEventCreate(&e1));
    fma_chain_kernel<R><<<blocks, threads, 0, c.stream>>>(out.p, iters, (R)0.999999, (R)1e-7);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep)
    {
        IBLGF_CUDA(cudaEventRecord(e0, c.stream));
        fma_chain_kernel<R><<<blocks, threads, 0, c.stream>>>(out.p, iters, (R)0.999999, (R)1e-7);
        IBLGF_CUDA(cudaEventRecord(e1, c.stream));
        IBLGF_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        IBLGF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = ms < best ? ms : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.launches += 4;
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}
}  // namespace

double measure_fma_peak(Ctx& c, int precision)
{
    return precision == IBLGF_FP32 ? run<float>(c) : run<double>(c);
}

}  // namespace iblgf_b200
