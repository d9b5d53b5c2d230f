// Device evaluation of the 7-point-Laplacian LGF, include/iblgf/lgf/
// lgf_gl_lookup.hpp:33-52 (table lookup with |n| sorted descending, returns
// -table) and :74-119 (3-term asymptotic expansion beyond N_max = 100; the
// third term only if some |n_i| < 600).
#pragma once

namespace iblgf_b200
{
constexpr int kLgfNmax = 100;

__host__ __device__ __forceinline__ int lgf_tidx(int x, int y, int z)
{
    return (x * (2 + 3 * x + x * x)) / 6 + y * (y + 1) / 2 + z;
}

__device__ __forceinline__ double lgf_asym_dev(int n1, int n2, int n3)
{
    const double a2 = (double)n1 * n1, b2 = (double)n2 * n2, c2 = (double)n3 * n3;
    const double r = sqrt(a2 + b2 + c2);
    const double a6 = a2 * a2 * a2, b6 = b2 * b2 * b2, c6 = c2 * c2 * c2;
    const double r6 = r * r * r * r * r * r;
    const double r7 = r6 * r, r13 = r6 * r6 * r;
    const double pi = 3.14159265358979323846;
    double g = -1.0 / 4.0 / pi / r;
    g -= (a2 * a2 + b2 * b2 + c2 * c2 - 3.0 * a2 * b2 - 3.0 * b2 * c2 - 3.0 * c2 * a2) / 16.0 / pi / r7;
    if (n1 < 600 || n2 < 600 || n3 < 600)
    {
        double t = -3.0 * (23.0 * (a6 * a2 + b6 * b2 + c6 * c2) -
                           244.0 * (b6 * c2 + c6 * b2 + a6 * b2 + b6 * a2 + a6 * c2 + c6 * a2) +
                           621.0 * (a2 * a2 * b2 * b2 + b2 * b2 * c2 * c2 + c2 * c2 * a2 * a2) -
                           228.0 * (a2 * a2 * b2 * c2 + a2 * b2 * b2 * c2 + a2 * b2 * c2 * c2));
        g += t / r13 / 4.0 * (8.0 / (768.0 * pi));
    }
    return g;
}

__device__ __forceinline__ double lgf_get_dev(int x, int y, int z, const double* __restrict__ table)
{
    x = abs(x);
    y = abs(y);
    z = abs(z);
    if (x <= kLgfNmax && y <= kLgfNmax && z <= kLgfNmax)
    {
        int a = x, b = y, c = z, t;
        if (a < b) { t = a; a = b; b = t; }
        if (a < c) { t = a; a = c; c = t; }
        if (b < c) { t = b; b = c; c = t; }
        return -__ldg(&table[lgf_tidx(a, b, c)]);
    }
    return lgf_asym_dev(x, y, z);
}

}  // namespace iblgf_b200
