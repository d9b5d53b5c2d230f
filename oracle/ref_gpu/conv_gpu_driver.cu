// Test and benchmark infrastructure: drives the reference's cuFFT block
// convolution (fft::Convolution_GPU<3>, include/iblgf/utilities/
// convolution_GPU.hpp:289-590) through its stock per-pair interface, the way
// Fmm::fmm_tt / compute_influence_field call it (include/iblgf/fmm/
// fmm.hpp:988-1027, 1167-1195): per target, apply_forward_add for every
// (source, LGF block) pair (batched FFTs of 10 sources, spectral product,
// sum), then apply_backward (scale, c2r, copy to the host, add the window
// into the target). The types it is templated on are stood in for here:
// a block descriptor (base, extent), a host DataField (real_block(),
// get_real_local) and an LGF kernel whose dft_gpu caches one device spectrum
// per key as LGF_Base::dft_gpu does (lgf.hpp:102-136), computed with the
// convolution's own dft_r2c.
//
//   ref_conv_gpu check <Nb> <in.bin> <out.bin>
//       in: kernel block (2Nb-1)^3 and source block Nb^3 doubles (x fastest);
//       out: the target block Nb^3 after one pair (scale 1)
//   ref_conv_gpu time <Nb> <targets> <pairs per target> <passes>
//       synthetic pairs (sources from a pool of 64 blocks, 343 distinct LGF
//       blocks cached after their first use); prints one JSON line with the
//       wall time per target of the timed passes (after one warm pass)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include <iblgf/utilities/convolution_GPU.hpp>

using iblgf::types::vector_type;
using dims_t = vector_type<int, 3>;

struct BlockDesc
{
    dims_t b, e;
    const dims_t& base() const { return b; }
    const dims_t& extent() const { return e; }
};

struct HostField
{
    int nb = 0;
    std::vector<double> v;
    BlockDesc rb;
    explicit HostField(int n)
    : nb(n)
    , v((size_t)n * n * n, 0.0)
    {
        rb.b = dims_t(0);
        rb.e = dims_t(n);
    }
    const BlockDesc& real_block() const { return rb; }
    const double& get_real_local(int i, int j, int k) const { return v[i + (size_t)nb * (j + (size_t)nb * k)]; }
    double& get_real_local(int i, int j, int k) { return v[i + (size_t)nb * (j + (size_t)nb * k)]; }
    // the 2-D form the templates also name (their 2-D branch is compiled, not run)
    double& get_real_local(int i, int j) { return v[i + (size_t)nb * j]; }
};

struct SpectrumEntry
{
    cufftDoubleComplex* device = nullptr;
    size_t size = 0;
};

// LGF kernel stand-in: one cached device spectrum per key
struct CachedKernel
{
    int P = 0;
    long long key = 0;
    std::map<long long, SpectrumEntry> cache;
    std::vector<double> block;  // values of the next uncached block (P^3)
    std::vector<double> (*fill)(long long key, int P) = nullptr;

    template<class Conv>
    SpectrumEntry* dft_gpu(const BlockDesc&, dims_t, Conv* conv, int)
    {
        auto it = cache.find(key);
        if (it != cache.end()) return &it->second;
        block = fill ? fill(key, P) : block;
        cufftDoubleComplex* d = conv->dft_r2c(block);
        SpectrumEntry e;
        e.size = conv->dft_r2c_size();
        cudaMalloc(&e.device, e.size * sizeof(cufftDoubleComplex));
        cudaMemcpy(e.device, d, e.size * sizeof(cufftDoubleComplex), cudaMemcpyDeviceToDevice);
        return &cache.emplace(key, e).first->second;
    }
    ~CachedKernel()
    {
        for (auto& kv : cache) cudaFree(kv.second.device);
    }
};

// smooth, LGF-like values of a synthetic kernel block (timing only)
std::vector<double> synthetic_block(long long key, int P)
{
    std::vector<double> v((size_t)P * P * P);
    const double off = 1.0 + (double)(key % 343);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i)
                v[i + (size_t)P * (j + (size_t)P * k)] =
                    -1.0 / (4.0 * M_PI * std::sqrt((i + off) * (i + off) + (double)j * j + (double)k * k + 1.0));
    return v;
}

// A runtime error recorded by the reference code's calls (some are benign,
// e.g. host-buffer registrations): printed; only a device fault fails the run.
int report_errors()
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return 0;
    std::fprintf(stderr, "ref_conv_gpu: CUDA runtime reported %s (%s)\n", cudaGetErrorName(e), cudaGetErrorString(e));
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    const std::string mode = argv[1];
    const int Nb = std::atoi(argv[2]), P = 2 * Nb - 1;
    if (Nb < 4 || Nb > 64) return 2;
    iblgf::fft::Convolution_GPU<3> conv(dims_t(Nb), dims_t(Nb), 10);
    BlockDesc extractor{dims_t(0), dims_t(Nb)};
    BlockDesc lgf_block{dims_t(0), dims_t(P)};
    if (mode == "check" && argc == 5)
    {
        FILE* fi = std::fopen(argv[3], "rb");
        if (!fi) return 2;
        CachedKernel k;
        k.P = P;
        k.block.resize((size_t)P * P * P);
        HostField src(Nb), tgt(Nb);
        const bool ok = std::fread(k.block.data(), 8, k.block.size(), fi) == k.block.size() &&
                        std::fread(src.v.data(), 8, src.v.size(), fi) == src.v.size();
        std::fclose(fi);
        if (!ok) return 2;
        conv.fft_backward_field_clean();
        conv.apply_forward_add(lgf_block, &k, 0, src);
        conv.apply_backward(extractor, tgt, 1.0);
        FILE* fo = std::fopen(argv[4], "wb");
        std::fwrite(tgt.v.data(), 8, tgt.v.size(), fo);
        std::fclose(fo);
        return report_errors();
    }
    if (mode == "time" && argc == 6)
    {
        const int T = std::atoi(argv[3]), Q = std::atoi(argv[4]), passes = std::atoi(argv[5]);
        if (T < 1 || Q < 1 || passes < 1) return 2;
        CachedKernel k;
        k.P = P;
        k.fill = synthetic_block;
        std::mt19937 rng(7);
        std::uniform_real_distribution<double> U(-1.0, 1.0);
        std::vector<HostField> pool;
        for (int s = 0; s < 64; ++s)
        {
            pool.emplace_back(Nb);
            for (double& x : pool.back().v) x = U(rng);
        }
        HostField tgt(Nb);
        double ms = 0.0;
        for (int pass = 0; pass <= passes; ++pass)  // pass 0 fills the spectrum cache
        {
            const auto t0 = std::chrono::steady_clock::now();
            for (int t = 0; t < T; ++t)
            {
                conv.fft_backward_field_clean();
                for (int q = 0; q < Q; ++q)
                {
                    k.key = ((long long)t * Q + q) % 343;
                    conv.apply_forward_add(lgf_block, &k, 0, pool[(t + q) % 64]);
                }
                conv.apply_backward(extractor, tgt, 1.0);
            }
            cudaDeviceSynchronize();
            const auto t1 = std::chrono::steady_clock::now();
            if (pass) ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        if (report_errors()) return 1;
        std::printf("{\"targets\": %d, \"pairs_per_target\": %d, \"passes\": %d, \"ms_per_target\": %.6f}\n", T, Q,
                    passes, ms / passes / T);
        return 0;
    }
    return 2;
}
