// LGF table generation on the device, FP64, and point evaluation.
//
// table(n1,n2,n3) = int_0^inf e^{-6t} I_n1(2t) I_n2(2t) I_n3(2t) dt for
// 0 <= n3 <= n2 <= n1 <= 100 — the quantity the reference tabulates offline
// (include/iblgf/lgf/lgf_table_gen/python_lgf.py:9-21 with scipy quad) and
// ships as src/lgf/lgf_gl_lookup.cpp. Here: composite 32-point Gauss-Legendre
// on octave intervals of [0, 1e4] plus the term-by-term integral of the
// product of the large-argument expansions e^{-x} I_n(x) ~ (2 pi x)^{-1/2}
// sum_k (-1)^k a_k(n) x^{-k} (Abramowitz & Stegun 9.7.1) on [1e4, inf).
// e^{-x} I_n(x) for all n at a node comes from Miller's backward recurrence
// I_{k-1} = I_{k+1} + (2k/x) I_k normalised by e^x = I_0 + 2 sum_k I_k
// (A&S 9.6.26 and 9.6.37), one thread per node.
#include <cmath>
#include <vector>

#include "ctx.hpp"
#include "lgf_dev.cuh"

namespace iblgf_b200
{
namespace
{
constexpr int kNgl = 32;
constexpr double kTmax = 1.0e4;
constexpr int kTail = 14;

void gauss_legendre_nodes(int n, std::vector<double>& x, std::vector<double>& w)
{
    x.resize(n);
    w.resize(n);
    for (int i = 0; i < n; ++i)
    {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it)
        {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k)
            {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k)
        {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// e^{-x} I_n(x), n = 0..kLgfNmax, at x = 2 t_q for every quadrature node q
__global__ void bessel_nodes_kernel(const double* __restrict__ t, int nq, double* __restrict__ F)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const double x = 2.0 * t[q];
    double* out = F + (size_t)q * (kLgfNmax + 1);
    const int m = kLgfNmax + 30 + (int)ceil(sqrt(90.0 * x));
    double a = 0.0, b = 1e-280, sum = 0.0;
    for (int n = 0; n <= kLgfNmax; ++n) out[n] = 0.0;
    for (int k = m; k >= 1; --k)
    {
        const double c = a + (2.0 * k / x) * b;
        sum += b;
        if (k <= kLgfNmax) out[k] = b;
        a = b;
        b = c;
        if (fabs(b) > 1e250)
        {
            a *= 1e-250;
            b *= 1e-250;
            sum *= 1e-250;
            for (int n = k; n <= kLgfNmax; ++n) out[n] *= 1e-250;
        }
    }
    out[0] = b;
    const double inv = 1.0 / (b + 2.0 * sum);
    for (int n = 0; n <= kLgfNmax; ++n) out[n] *= inv;
}

// one block per n1; threads over (n2, n3) with n3 <= n2 <= n1
__global__ void table_kernel(const double* __restrict__ F, const double* __restrict__ w, int nq,
                             double* __restrict__ table)
{
    const int n1 = blockIdx.x;
    const int npairs = (n1 + 1) * (n1 + 2) / 2;
    __shared__ double a1[kTail + 1];
    if (threadIdx.x == 0)
    {
        double a = 1.0;
        a1[0] = 1.0;
        for (int k = 1; k <= kTail; ++k)
        {
            a *= -(4.0 * n1 * n1 - (2.0 * k - 1.0) * (2.0 * k - 1.0)) / (8.0 * k);
            a1[k] = a;
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < npairs; p += blockDim.x)
    {
        int n2 = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
        while (n2 * (n2 + 1) / 2 > p) --n2;
        while ((n2 + 1) * (n2 + 2) / 2 <= p) ++n2;
        const int n3 = p - n2 * (n2 + 1) / 2;
        double s = 0.0;
        for (int q = 0; q < nq; ++q)
        {
            const double* fq = F + (size_t)q * (kLgfNmax + 1);
            s += w[q] * __ldg(fq + n1) * __ldg(fq + n2) * __ldg(fq + n3);
        }
        double a2[kTail + 1], a3[kTail + 1];
        double aa = 1.0, bb = 1.0;
        a2[0] = a3[0] = 1.0;
        for (int k = 1; k <= kTail; ++k)
        {
            aa *= -(4.0 * n2 * n2 - (2.0 * k - 1.0) * (2.0 * k - 1.0)) / (8.0 * k);
            bb *= -(4.0 * n3 * n3 - (2.0 * k - 1.0) * (2.0 * k - 1.0)) / (8.0 * k);
            a2[k] = aa;
            a3[k] = bb;
        }
        double tail = 0.0;
        for (int m = 0; m <= kTail; ++m)
        {
            double cm = 0.0;
            for (int i = 0; i <= m; ++i)
                for (int j = 0; j <= m - i; ++j) cm += a1[i] * a2[j] * a3[m - i - j];
            tail += cm * exp2(-(double)m) * pow(kTmax, -0.5 - m) / (m + 0.5);
        }
        tail *= pow(4.0 * 3.14159265358979323846, -1.5);
        table[lgf_tidx(n1, n2, n3)] = s + tail;
    }
}

__global__ void lgf_eval_kernel(const int* __restrict__ xyz, size_t n, const double* __restrict__ table,
                                double* __restrict__ out)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = lgf_get_dev(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], table);
}
}  // namespace

void launch_lgf_table(Ctx& c)
{
    std::vector<double> gx, gw;
    gauss_legendre_nodes(kNgl, gx, gw);
    std::vector<double> edges{0.0};
    for (double e = 0.125; e < kTmax; e *= 2.0) edges.push_back(e);
    edges.push_back(kTmax);
    std::vector<double> t, w;
    for (size_t i = 0; i + 1 < edges.size(); ++i)
        for (int j = 0; j < kNgl; ++j)
        {
            const double a = edges[i], b = edges[i + 1];
            t.push_back(0.5 * (b - a) * gx[j] + 0.5 * (b + a));
            w.push_back(0.5 * (b - a) * gw[j]);
        }
    const int nq = (int)t.size();
    DevBuf<double> dt, dw, dF;
    dt.upload(t, c.stream);
    dw.upload(w, c.stream);
    dF.alloc((size_t)nq * (kLgfNmax + 1));
    c.d_lgf_table.alloc(lgf_tidx(kLgfNmax, kLgfNmax, kLgfNmax) + 1);
    bessel_nodes_kernel<<<(nq + 63) / 64, 64, 0, c.stream>>>(dt.p, nq, dF.p);
    table_kernel<<<kLgfNmax + 1, 256, 0, c.stream>>>(dF.p, dw.p, nq, c.d_lgf_table.p);
    c.launches += 2;
    IBLGF_CUDA(cudaGetLastError());
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

namespace
{
// LGF_GE::get (lgf_ge.hpp:95-110): E(n; alpha) = f[|n1|] f[|n2|] f[|n3|],
// f[k] = e^{-2 alpha} I_k(2 alpha) from the context's table of this alpha;
// offsets past the table (|n_i| >= stride, f below 1e-300 there for the
// alphas of a time step) give 0
__global__ void lgf_ge_eval_kernel(const int* __restrict__ xyz, size_t n, const double* __restrict__ f, int stride,
                                   double* __restrict__ out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = abs(xyz[3 * i]), b = abs(xyz[3 * i + 1]), d = abs(xyz[3 * i + 2]);
    out[i] = (a < stride && b < stride && d < stride) ? f[a] * f[b] * f[d] : 0.0;
}
}  // namespace

void launch_lgf_ge_eval(Ctx& c, int ge, const int* d_coords, size_t n, double* d_out)
{
    if (!n) return;
    lgf_ge_eval_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(
        d_coords, n, c.d_ge.p + (size_t)ge * c.ge_stride, c.ge_stride, d_out);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void launch_lgf_eval(Ctx& c, const int* d_coords, size_t n, double* d_out)
{
    if (!n) return;
    lgf_eval_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d_coords, n, c.d_lgf_table.p, d_out);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

}  // namespace iblgf_b200
