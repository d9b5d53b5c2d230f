// ORACLE (test infrastructure): complex FFT of arbitrary length by recursive
// mixed-radix decimation in time, each prime factor by a direct DFT. It stands
// in for the FFTW plans of src/utilities/convolution.cpp:25-238 (the reference
// uses unnormalised FFTW r2c/c2r transforms; so does this code).
#include <cmath>

#include "orc.hpp"

namespace orc
{
Fft1d::Fft1d(int n_)
: n(n_)
{
    int m = n;
    for (int p = 2; p * p <= m; ++p)
        while (m % p == 0)
        {
            factors.push_back(p);
            m /= p;
        }
    if (m > 1) factors.push_back(m);
    tw_fwd.resize(n);
    tw_bwd.resize(n);
    for (int j = 0; j < n; ++j)
    {
        const double a = 2.0 * M_PI * (double)j / (double)n;
        tw_fwd[j] = cplx(std::cos(a), -std::sin(a));
        tw_bwd[j] = cplx(std::cos(a), std::sin(a));
    }
}

namespace
{
// out[k] = sum_j in[j*stride] w^{j k}, length len = product of factors[f..]
void rec(const cplx* in, int istride, cplx* out, int len, const std::vector<int>& fac,
         int f, const std::vector<cplx>& tw, int n, cplx* work)
{
    if (len == 1)
    {
        out[0] = in[0];
        return;
    }
    const int p = fac[f];
    const int m = len / p;
    // sub-transforms of the p decimated sequences, stored consecutively
    for (int r = 0; r < p; ++r)
        rec(in + r * istride, istride * p, work + r * m, m, fac, f + 1, tw, n, out);
    const int tstep = n / len;  // twiddle index unit for length len
    for (int k = 0; k < m; ++k)
    {
        for (int q = 0; q < p; ++q)
        {
            const int kk = k + q * m;
            cplx s = 0.0;
            for (int r = 0; r < p; ++r)
            {
                const int e = (int)(((long long)r * kk) % len) * tstep;
                s += work[r * m + k] * tw[e];
            }
            out[kk] = s;
        }
    }
}
}  // namespace

void Fft1d::run(cplx* x, int stride, bool forward, cplx* work) const
{
    // work must hold 3*n entries
    cplx* in = work;
    cplx* out = work + n;
    cplx* scratch = work + 2 * n;
    for (int j = 0; j < n; ++j) in[j] = x[j * stride];
    // the recursion ping-pongs between out and scratch; copy through a
    // private buffer to keep levels independent
    std::vector<cplx> tmp(n);
    rec(in, 1, out, n, factors, 0, forward ? tw_fwd : tw_bwd, n, tmp.data());
    (void)scratch;
    for (int j = 0; j < n; ++j) x[j * stride] = out[j];
}

}  // namespace orc
