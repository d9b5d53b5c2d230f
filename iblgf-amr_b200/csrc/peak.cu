// Throughput probes for roofline denominators the driver-measured peaks (HBM
// copy, bf16 GEMM) do not cover:
//  * FMA chains: the FP64 / FP32 CUDA-core peak. Each thread runs 8
//    independent register-resident FMA chains; grid = 8 CTAs per SM.
//  * tensor-core issue rate: SM clocks per tcgen05.mma kind::tf32 of shape
//    M = 128, K = 8 and a given N (A in tensor memory, B in shared memory),
//    issued back to back by one thread per CTA, one CTA per SM, into a few
//    independent accumulators. The tensor-core spectral MAC issues N = 16
//    products; this rate bounds it.
#include <algorithm>
#include <vector>

#include "ctx.hpp"
#include "tcgen05.cuh"

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
// The bounded-wait path of the kernels that wait on mbarriers, run on
// purpose: one CTA waits on a barrier that nothing arrives on, `polls`
// try_wait polls, then records the timeout in the status word and returns.
__global__ void wait_selftest_kernel(long long polls, int* status)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    const bool ok = mbar_wait(&bar, 0, polls);
    if (!ok && threadIdx.x == 0) atomicOr(status, kStatusTimeout);
}

template<int N, int NACC>
__global__ void __launch_bounds__(128) tc_rate_kernel(int reps, long long* out, int* status)
{
    static_assert(NACC * N <= 448, "accumulator columns below the A columns");
    __shared__ __align__(1024) float bs[N * 8];
    __shared__ __align__(8) unsigned long long bar;
    __shared__ unsigned tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int i = tid; i < N * 8; i += blockDim.x) bs[i] = 0.0f;
    if (warp == 0) tc::alloc(&tmem, 512);
    if (tid == 0) mbar_init(&bar, 1);
    fence_proxy_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const unsigned tb = tmem;
    long long t0 = 0;
    if (tid == 0)
    {
        constexpr unsigned idesc = tc::idesc_tf32(128, N);
        const unsigned long long bd = tc::smem_desc(bs);
        t0 = clock64();
        for (int r = 0; r < reps; ++r)
            tc::mma_tf32(tb + (unsigned)((r % NACC) * N), tb + 448u, bd, idesc, r >= NACC);
        tc::commit(&bar);
    }
    const bool ok = mbar_wait(&bar, 0);
    if (tid == 0)
    {
        if (!ok) atomicOr(status, kStatusTimeout);
        out[blockIdx.x] = clock64() - t0;
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc::fence_after();
        tc::dealloc(tb, 512);
    }
}

template<int N, int NACC>
double tc_rate(Ctx& c)
{
    int dev = 0, sms = 0;
    IBLGF_CUDA(cudaGetDevice(&dev));
    IBLGF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DevBuf<long long> out;
    out.alloc(sms);
    const int reps = 4096;
    double best = 1e30;
    for (int rep = 0; rep < 2; ++rep)  // the first run warms up
    {
        tc_rate_kernel<N, NACC><<<sms, 128, 0, c.stream>>>(reps, out.p, c.d_status.p);
        IBLGF_CUDA(cudaGetLastError());
        std::vector<long long> h(sms);
        IBLGF_CUDA(cudaMemcpyAsync(h.data(), out.p, sms * sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        double sum = 0;
        for (long long v : h) sum += (double)v;
        best = std::min(best, sum / sms / reps);
    }
    c.launches += 2;
    return best;
}
}  // namespace

void wait_selftest(Ctx& c, long long polls)
{
    if (polls < 1 || polls > kWaitLimit) throw Error(IBLGF_EINVAL, "polls must be in [1, 2^22]");
    wait_selftest_kernel<<<1, 32, 0, c.stream>>>(polls, c.d_status.p);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

double measure_tc_rate(Ctx& c, int n)
{
    switch (n)
    {
        case 16: return tc_rate<16, 4>(c);
        case 32: return tc_rate<32, 4>(c);
        case 64: return tc_rate<64, 4>(c);
        case 128: return tc_rate<128, 2>(c);
        case 256: return tc_rate<256, 1>(c);
        default: throw Error(IBLGF_EINVAL, "N must be 16, 32, 64, 128 or 256");
    }
}

double measure_fma_peak(Ctx& c, int precision)
{
    return precision == IBLGF_FP32 ? run<float>(c) : run<double>(c);
}

}  // namespace iblgf_b200
