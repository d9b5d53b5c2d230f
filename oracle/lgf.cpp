// ORACLE (test infrastructure): lattice Green's function of the 7-point
// Laplacian. Restates include/iblgf/lgf/lgf_gl_lookup.hpp (get :33-52, asym
// :74-119) and regenerates the table that the reference ships as the missing
// src/lgf/lgf_gl_lookup.cpp, following lgf_table_gen/python_lgf.py:9-21 and
// lgf_integrator.py:7-27:
//     table(n1,n2,n3) = int_0^inf e^{-6t} I_n1(2t) I_n2(2t) I_n3(2t) dt,
//     n1 >= n2 >= n3, 0..100, get() returns -table.
// Method (own): composite Gauss-Legendre on octave intervals of [0, 1e4]
// plus the integral of the product of the large-argument asymptotic series of
// e^{-x} I_n(x) (Abramowitz & Stegun 9.7.1) on [1e4, inf). The scaled Bessel
// functions of all orders come from Miller's backward recurrence normalised by
// e^{x} = I_0 + 2 sum_k I_k (A&S 9.6.26, 9.6.37).
#include <algorithm>
#include <cmath>
#include <mutex>

#include "orc.hpp"

namespace orc
{
namespace
{
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w)
{
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i)
    {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it)
        {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k)
            {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const double dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k)
        {
            double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        const double dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

inline int tidx(int x, int y, int z)
{
    return (x * (2 + 3 * x + x * x)) / 6 + y * (y + 1) / 2 + z;
}

std::vector<double> g_table;
std::once_flag g_once;

void build_table()
{
    const int N = kLgfNmax;
    const double T = 1.0e4;
    const int ngl = 32;
    std::vector<double> gx, gw;
    gauss_legendre(ngl, gx, gw);
    std::vector<double> edges{0.0};
    for (double e = 0.125; e < T; e *= 2.0) edges.push_back(e);
    edges.push_back(T);
    const int nint = (int)edges.size() - 1;
    const int nq = nint * ngl;
    std::vector<double> wq(nq);
    std::vector<double> f((size_t)nq * (N + 1));  // f[q*(N+1)+n]
#pragma omp parallel for schedule(dynamic)
    for (int q = 0; q < nq; ++q)
    {
        const int iv = q / ngl, j = q % ngl;
        const double a = edges[iv], b = edges[iv + 1];
        const double t = 0.5 * (b - a) * gx[j] + 0.5 * (b + a);
        wq[q] = 0.5 * (b - a) * gw[j];
        bessel_ie_all(2.0 * t, N, &f[(size_t)q * (N + 1)]);
    }
    // asymptotic coefficients a'_k(n) = (-1)^k prod_j (4n^2-(2j-1)^2)/(k! 8^k)
    const int K = 14;
    std::vector<double> ac((size_t)(N + 1) * (K + 1));
    for (int n = 0; n <= N; ++n)
    {
        double a = 1.0;
        ac[(size_t)n * (K + 1)] = 1.0;
        for (int k = 1; k <= K; ++k)
        {
            a *= -(4.0 * n * n - (2.0 * k - 1.0) * (2.0 * k - 1.0)) / (8.0 * k);
            ac[(size_t)n * (K + 1) + k] = a;
        }
    }
    g_table.assign(tidx(N, N, N) + 1, 0.0);
#pragma omp parallel for schedule(dynamic)
    for (int n1 = 0; n1 <= N; ++n1)
    {
        for (int n2 = 0; n2 <= n1; ++n2)
        {
            for (int n3 = 0; n3 <= n2; ++n3)
            {
                double s = 0.0;
                for (int q = 0; q < nq; ++q)
                {
                    const double* fq = &f[(size_t)q * (N + 1)];
                    s += wq[q] * fq[n1] * fq[n2] * fq[n3];
                }
                // tail: (4 pi t)^{-3/2} sum_m c_m (2t)^{-m}
                double c12[2 * K + 1] = {0};
                for (int i = 0; i <= K; ++i)
                    for (int j = 0; j <= K; ++j)
                        c12[i + j] += ac[(size_t)n1 * (K + 1) + i] *
                                      ac[(size_t)n2 * (K + 1) + j];
                double tail = 0.0;
                for (int m = 0; m <= K; ++m)
                {
                    double cm = 0.0;
                    for (int i = 0; i <= m; ++i)
                        cm += c12[i] * ac[(size_t)n3 * (K + 1) + (m - i)];
                    tail += cm * std::pow(2.0, -m) * std::pow(T, -0.5 - m) / (m + 0.5);
                }
                tail *= std::pow(4.0 * M_PI, -1.5);
                g_table[tidx(n1, n2, n3)] = s + tail;
            }
        }
    }
}
}  // namespace

void bessel_ie_all(double x, int nmax, double* out)
{
    if (x == 0.0)
    {
        // e^0 I_n(0): 1 for n = 0, 0 otherwise (the recurrence divides by x)
        for (int n = 0; n <= nmax; ++n) out[n] = n == 0 ? 1.0 : 0.0;
        return;
    }
    const int m = std::max(nmax, 0) + 30 + (int)std::ceil(std::sqrt(90.0 * x));
    double a = 0.0, b = 1e-280, sum = 0.0;
    for (int n = 0; n <= nmax; ++n) out[n] = 0.0;
    for (int k = m; k >= 1; --k)
    {
        const double c = a + (2.0 * k / x) * b;  // I_{k-1}
        sum += b;
        if (k <= nmax) out[k] = b;
        a = b;
        b = c;
        if (std::fabs(b) > 1e250)
        {
            a *= 1e-250;
            b *= 1e-250;
            sum *= 1e-250;
            for (int n = k; n <= nmax; ++n) out[n] *= 1e-250;
        }
    }
    out[0] = b;
    const double norm = b + 2.0 * sum;
    for (int n = 0; n <= nmax; ++n) out[n] /= norm;
}

int lgf_table_size() { return tidx(kLgfNmax, kLgfNmax, kLgfNmax) + 1; }

const std::vector<double>& lgf_table()
{
    std::call_once(g_once, build_table);
    return g_table;
}

double lgf_asym(int n1, int n2, int n3)
{
    const double a2 = (double)n1 * n1, b2 = (double)n2 * n2, c2 = (double)n3 * n3;
    const double r = std::sqrt(a2 + b2 + c2);
    const double a6 = a2 * a2 * a2, b6 = b2 * b2 * b2, c6 = c2 * c2 * c2;
    const double a8 = a6 * a2, b8 = b6 * b2, c8 = c6 * c2;
    const double r6 = r * r * r * r * r * r;
    const double r7 = r6 * r, r13 = r6 * r6 * r;
    double g = -1.0 / 4.0 / M_PI / r;
    g -= (a2 * a2 + b2 * b2 + c2 * c2 - 3.0 * a2 * b2 - 3.0 * b2 * c2 - 3.0 * c2 * a2) /
         16.0 / M_PI / r7;
    if (n1 < 600 || n2 < 600 || n3 < 600)
    {
        const double coef = 8.0 / (768.0 * M_PI);
        double t = -3.0 * (23 * (a8 + b8 + c8) -
                           244 * (b6 * c2 + c6 * b2 + a6 * b2 + b6 * a2 + a6 * c2 + c6 * a2) +
                           621 * ((a2 * a2) * (b2 * b2) + (b2 * b2) * (c2 * c2) +
                                  (c2 * c2) * (a2 * a2)) -
                           228 * ((a2 * a2) * b2 * c2 + a2 * (b2 * b2) * c2 +
                                  a2 * b2 * (c2 * c2)));
        t = t / r13 / 4.0 * coef;
        g += t;
    }
    return g;
}

double lgf_get(int x, int y, int z)
{
    x = std::abs(x);
    y = std::abs(y);
    z = std::abs(z);
    if (x <= kLgfNmax && y <= kLgfNmax && z <= kLgfNmax)
    {
        if (x < y) std::swap(x, y);
        if (x < z) std::swap(x, z);
        if (y < z) std::swap(y, z);
        return -lgf_table()[tidx(x, y, z)];
    }
    return lgf_asym(x, y, z);
}

}  // namespace orc
