// Two-dimensional Helmholtz lattice Green's function (the kernel of the
// reference's Fourier-in-z solvers, one per z mode) and the uniform 2-D
// screened Poisson solve built on it.
//
// Helmholtz_Lookup (include/iblgf/lgf/helmholtz_lookup.hpp:45-176) and
// Helmholtz<2>::get (include/iblgf/lgf/helmholtz.hpp:152-163): for the
// offset (n, m), |n| >= |m| after the swap,
//     G_c(n, m) = 1/(2 pi) int_{-pi}^{pi} (1 - cos(m x) K(x)^-|n|) / (K - 1/K) dx,
//     a = 4 - 2 cos x + c^2,  K = (a + sqrt(a^2 - 4)) / 2,
// and get() returns G_c(n, m) - origin(c), origin(c) = 1/(2 pi) int 1/(K - 1/K)
// = 0.5 / (2 + c^2/2) 2F1(1/2, 1/2; 1; (2 / (2 + c^2/2))^2) (origin_val, the
// Gauss series summed to 1e-20). So get(n, m) = -1/(2 pi) int cos(m x)
// K^-|n| / (K - 1/K) dx, the decaying solution of the five-point screened
// Poisson equation g(n+1,m) + g(n-1,m) + g(n,m+1) + g(n,m-1) - (4 + c^2) g(n,m)
// = delta_{n,m}. The integrand is periodic and analytic in a strip of
// half-width ~ c around the real axis, so the trapezoidal rule with N points
// converges like e^{-c N}; the reference refines a trapezoidal rule to a
// relative change of 1e-20 (boost::math::quadrature::trapezoidal). Here N is
// fixed per c (a power of two with c N >= 48, at least 64): relative error
// below 1e-16 for c >= ~0.01.
//
// Mode 0 (c = 0) is the 2-D lattice Green's function of the five-point
// Laplacian, LGF_GL<2> (lgf_gl.hpp:93-99, lgf_gl_lookup.hpp:46-60, 121-131):
// the reference reads it from a table for small offsets (not in the reference
// tree) and uses -asym(n, m) = log(r) / (2 pi) - Cfund - Integral_val -
// cos(4 theta) / (24 pi r^2) beyond; both are the regularised LGF
//     G0(n, m) = 1/pi int_0^pi (1 - e^{-|n| s} cos(m x)) / (2 sinh s) dx,
//     cosh s = 2 - cos x,
// with G0(0, 0) = 0 and Delta_h G0 = delta. Its integrand is smooth on
// [0, pi] but has a |x| kink when continued to [-pi, pi], so G0 uses
// Gauss-Legendre nodes on [0, pi] (Newton iteration on the Legendre
// recurrence, computed on the host) instead of the periodic trapezoidal rule.
//
// helm2d_table_kernel  get(n, m) for 0 <= n < nx, 0 <= m < ny (one thread each)
// helm2d_apply_kernel  u(i) = sum_j get(i - j) f(j) over a uniform nx x ny
//                      cell grid, one thread per target cell, the source row
//                      staged through shared memory
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "ctx.hpp"

namespace iblgf_b200
{
namespace
{
// A set of up to 2048 units (z modes or z planes), passed by value.
struct UnitMask
{
    static constexpr int kMax = 2048;
    unsigned w[kMax / 32];
    __device__ bool on(int i) const { return (w[i >> 5] >> (i & 31)) & 1u; }
};

// Offset of element i: (i % nx, i / nx) of a table, or the i-th pair of nm
// (absolute values) when a list of offsets is given.
__device__ inline void offset_of(int i, int nx, const int* nm, int& n, int& m)
{
    if (nm)
    {
        n = abs(nm[2 * i]);
        m = abs(nm[2 * i + 1]);
    }
    else
    {
        n = i % nx;
        m = i / nx;
    }
}

__global__ void helm2d_table_kernel(int nx, int ny, const int* __restrict__ nm, double c, int npts,
                                    double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    int n, m;
    offset_of(i, nx, nm, n, m);
    if (n < m)
    {
        const int t = n;
        n = m;
        m = t;
    }
    const double h = 2.0 * M_PI / npts;
    double s = 0.0;
    for (int k = 0; k < npts; ++k)
    {
        const double x = -M_PI + h * k;
        const double a = 4.0 - 2.0 * cos(x) + c * c;
        const double K = 0.5 * (a + sqrt(a * a - 4.0));
        s += cos(m * x) * pow(K, -(double)n) / (K - 1.0 / K);
    }
    out[i] = -s * h / (2.0 * M_PI);
}

__global__ void lap2d_table_kernel(int nx, int ny, const int* __restrict__ nm, const double* __restrict__ gx,
                                   const double* __restrict__ gw, int npts, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    int n, m;
    offset_of(i, nx, nm, n, m);
    if (n < m)
    {
        const int t = n;
        n = m;
        m = t;
    }
    double s = 0.0;
    for (int k = 0; k < npts; ++k)
    {
        const double x = gx[k];
        const double hs = sin(0.5 * x);
        const double t = 2.0 * hs * hs;           // 1 - cos x without cancellation
        const double r = sqrt(t * (2.0 + t));     // sinh s
        const double sg = log1p(t + r);           // s = acosh(2 - cos x)
        s += gw[k] * (1.0 - exp(-n * sg) * cos(m * x)) / (2.0 * r);
    }
    out[i] = s / M_PI;
}

// u[y][x] += scale * sum over sources of table[|dy|][|dx|] f[sy][sx]
__global__ void helm2d_apply_kernel(int nx, int ny, const double* __restrict__ table, const double* __restrict__ f,
                                    double* __restrict__ u, double scale)
{
    extern __shared__ double srow[];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    double acc = 0.0;
    for (int sy = 0; sy < ny; ++sy)
    {
        __syncthreads();
        for (int i = threadIdx.x; i < nx; i += blockDim.x) srow[i] = f[(size_t)sy * nx + i];
        __syncthreads();
        if (x < nx)
        {
            const double* trow = table + (size_t)abs(y - sy) * nx;
            for (int sx = 0; sx < nx; ++sx) acc = fma(trow[abs(x - sx)], srow[sx], acc);
        }
    }
    if (x < nx) u[(size_t)y * nx + x] += scale * acc;
}

// Complex Helmholtz (Fourier-in-z) block operators on 2-D blocks
// (include/iblgf/operators/operators.hpp:1516-1545 laplace, :1585-1614
// gradient, :1763-1795 divergence, :1972-2008 curl, :2178-2217
// curl_transpose, the all-modes forms): a block holds [component][NB][NB],
// x fastest; a scalar field has sep = 2 N_modes components (mode i: real 2i,
// imaginary 2i+1), a vector field three groups of sep (x, y, z); the z
// derivative of mode i is multiplication by i omega_i, omega_i = 2 pi i / lz.
// One CTA per block, threads over (mode, interior node) pairs (nodes
// 1 .. NB-2 per axis); buffers are read, not written. The mask selects the modes written: all of
// them for the forms above, one for the _oneMode forms (:1548, :1620, :1801,
// :2017, :2224), the first N_modes / 2^r for the _refined forms (:1653,
// :1839, :2125), any set for the ModesBool forms (:1889, :1931); the
// components of unselected modes are left as they were.
// op: 0 laplace (cell -> cell), 1 gradient (cell -> face), 2 divergence
// (face -> cell), 3 curl (face -> edge), 4 curl_transpose (edge -> face, x scale)
template<int OP>
__global__ void helm_op_kernel(int nb, int n_modes, int in_comp, int out_comp, double dx, double lz, double scale,
                               UnitMask mask, const double* __restrict__ src, double* __restrict__ dst)
{
    const int sep = 2 * n_modes, N2 = nb * nb;
    const double* s = src + (size_t)blockIdx.x * in_comp * N2;
    double* d = dst + (size_t)blockIdx.x * out_comp * N2;
    const double fac = 1.0 / dx;
    // one thread per (mode, node): it owns every output component of that
    // mode at that node (consecutive threads take consecutive nodes)
    for (int q = threadIdx.x; q < n_modes * N2; q += blockDim.x)
    {
        const int mode = q / N2, p = q - mode * N2;
        const int x = p % nb, y = p / nb;
        if (x == 0 || y == 0 || x == nb - 1 || y == nb - 1 || !mask.on(mode)) continue;
        auto at = [&](int c, int ox, int oy) { return s[(size_t)c * N2 + p + ox + oy * nb]; };
        auto out = [&](int c) -> double& { return d[(size_t)c * N2 + p]; };
        const int re = 2 * mode, im = 2 * mode + 1;
        for (int i = re; i <= im; ++i)
        {
            if (OP == 0)
                out(i) = fac * fac * (-4.0 * at(i, 0, 0) + at(i, 0, -1) + at(i, 0, 1) + at(i, -1, 0) + at(i, 1, 0));
            else if (OP == 1)
            {
                out(i) = fac * (at(i, 0, 0) - at(i, -1, 0));
                out(sep + i) = fac * (at(i, 0, 0) - at(i, 0, -1));
            }
            else if (OP == 2)
                out(i) = fac * (-at(i, 0, 0) - at(sep + i, 0, 0) + at(i, 1, 0) + at(sep + i, 0, 1));
            else if (OP == 3)
            {
                out(i) = fac * (at(2 * sep + i, 0, 0) - at(2 * sep + i, 0, -1));
                out(sep + i) = fac * (-at(2 * sep + i, 0, 0) + at(2 * sep + i, -1, 0));
                out(2 * sep + i) = fac * (at(sep + i, 0, 0) - at(sep + i, -1, 0) - at(i, 0, 0) + at(i, 0, -1));
            }
            else
            {
                const double f = fac * scale;
                out(i) = f * (-at(2 * sep + i, 0, 0) + at(2 * sep + i, 0, 1));
                out(sep + i) = f * (at(2 * sep + i, 0, 0) - at(2 * sep + i, 1, 0));
                out(2 * sep + i) = f * (-at(sep + i, 0, 0) + at(sep + i, 1, 0) + at(i, 0, 0) - at(i, 0, 1));
            }
        }
        {
            const double om = 2.0 * M_PI * mode / lz;
            if (OP == 0)
            {
                out(re) -= at(re, 0, 0) * om * om;
                out(im) -= at(im, 0, 0) * om * om;
            }
            else if (OP == 1)
            {
                out(2 * sep + re) = -at(im, 0, 0) * om;
                out(2 * sep + im) = at(re, 0, 0) * om;
            }
            else if (OP == 2)
            {
                out(re) -= at(2 * sep + im, 0, 0) * om;
                out(im) += at(2 * sep + re, 0, 0) * om;
            }
            else
            {
                const double w = OP == 3 ? om : om * scale;
                out(re) += at(sep + im, 0, 0) * w;
                out(im) -= at(sep + re, 0, 0) * w;
                out(sep + re) -= at(im, 0, 0) * w;
                out(sep + im) += at(re, 0, 0) * w;
            }
        }
    }
}

// nonlinear_helmholtz (operators.hpp:2627-2766; _oneMode :2776-2831,
// _refined :2840-2895): the convective term on the z collocation planes of
// the Fourier-in-z solver. face (velocity), edge (vorticity) and dst are
// [block][3 n_planes][NB][NB] (x fastest; component group x, y, z, one
// component per z plane); per selected plane, at the interior nodes,
//   dst_x = 1/2 w_y (u_z + u_z[-x]) - 1/4 (w_z (u_y + u_y[-x]) + w_z[+y] (u_y[+y] + u_y[-x+y]))
//   dst_y = 1/4 (w_z (u_x + u_x[-y]) + w_z[+x] (u_x[+x] + u_x[+x-y])) - 1/2 w_x (u_z + u_z[-y])
//   dst_z = 1/2 (w_x u_y + w_x[+y] u_y[+y] - w_y u_x - w_y[+x] u_x[+x]).
// The mask selects planes: every plane; planes mode P .. mode P + P - 1 for
// the _oneMode form (P planes per mode); every 2^r-th for the _refined form.
__global__ void helm_nonlinear_kernel(int nb, int n_planes, UnitMask mask, const double* __restrict__ face,
                                      const double* __restrict__ edge, double* __restrict__ dst)
{
    const int N2 = nb * nb;
    const size_t blk = (size_t)blockIdx.x * 3 * n_planes * N2;
    const double* u = face + blk;
    const double* w = edge + blk;
    double* d = dst + blk;
    for (int q = threadIdx.x; q < n_planes * N2; q += blockDim.x)
    {
        const int i = q / N2, p = q - i * N2;
        const int x = p % nb, y = p / nb;
        if (x == 0 || y == 0 || x == nb - 1 || y == nb - 1 || !mask.on(i)) continue;
        const int cx = i, cy = n_planes + i, cz = 2 * n_planes + i;
        auto U = [&](int c, int ox, int oy) { return u[(size_t)c * N2 + p + ox + oy * nb]; };
        auto W = [&](int c, int ox, int oy) { return w[(size_t)c * N2 + p + ox + oy * nb]; };
        d[(size_t)cx * N2 + p] = 0.5 * W(cy, 0, 0) * (U(cz, 0, 0) + U(cz, -1, 0)) -
                                 0.25 * (W(cz, 0, 0) * (U(cy, 0, 0) + U(cy, -1, 0)) +
                                         W(cz, 0, 1) * (U(cy, 0, 1) + U(cy, -1, 1)));
        d[(size_t)cy * N2 + p] = 0.25 * (W(cz, 0, 0) * (U(cx, 0, 0) + U(cx, 0, -1)) +
                                         W(cz, 1, 0) * (U(cx, 1, 0) + U(cx, 1, -1))) -
                                 0.5 * W(cx, 0, 0) * (U(cz, 0, 0) + U(cz, 0, -1));
        d[(size_t)cz * N2 + p] = 0.5 * (W(cx, 0, 0) * U(cy, 0, 0) + W(cx, 0, 1) * U(cy, 0, 1) -
                                        W(cy, 0, 0) * U(cx, 0, 0) - W(cy, 1, 0) * U(cx, 1, 0));
    }
}

// Real-valued 2-D block operators of the Fourier-in-z family (fields in
// physical z, or one real mode; a, b inputs, d and e outputs, each
// [block][components][NB][NB], x fastest, with a_comp / b_comp / d_comp
// components; interior nodes written):
//  0 curl_helmholtz (operators.hpp:2305-2414): face -> edge on np z planes
//    (3 np components each); in-plane differences / dx_level, the z
//    difference between plane i and i - 1 (periodic) / dx_fine
//  1 curl_helmholtz_real (:2059-2081): face -> edge, edge x and y zero
//  2 curl_helmholtz_real with Uz (:2083-2119): edge x, y from the scalar b
//  3 curl_transpose_helmholtz_complex_linear (:2272-2303): edge -> face x, y
//    (d) and face z (e), scaled, plus the c scale cross terms
//  4 nonlinear_linear_helm (:2534-2572): face a, edge b -> face x, y (d) and
//    the z component (e) of the linearised convective term
//  5 curl_transpose, two-dimensional branch (:2416-2453): edge scalar ->
//    face x, y, scaled
template<int OP>
__global__ void helm_real_op_kernel(int nb, int np, double dx, double dx_fine, double c, double scale,
                                    const double* __restrict__ a, int a_comp, const double* __restrict__ b,
                                    int b_comp, double* __restrict__ d, int d_comp, double* __restrict__ e)
{
    const int N2 = nb * nb;
    const size_t blk = blockIdx.x;
    const double* A = a + blk * a_comp * N2;
    const double* Bf = b ? b + blk * b_comp * N2 : nullptr;
    double* D = d + blk * d_comp * N2;
    double* Ef = e ? e + blk * N2 : nullptr;
    const double fac = 1.0 / dx;
    const int units = OP == 0 ? np : 1;
    for (int q = threadIdx.x; q < units * N2; q += blockDim.x)
    {
        const int i = q / N2, p = q - i * N2;
        const int x = p % nb, y = p / nb;
        if (x == 0 || y == 0 || x == nb - 1 || y == nb - 1) continue;
        auto at = [&](int k, int ox, int oy) { return A[(size_t)k * N2 + p + ox + oy * nb]; };
        auto bt = [&](int k, int ox, int oy) { return Bf[(size_t)k * N2 + p + ox + oy * nb]; };
        auto out = [&](int k) -> double& { return D[(size_t)k * N2 + p]; };
        if (OP == 0)
        {
            // plane 0's z difference wraps to plane np - 1; its z component is
            // written as two differences (the reference's i = 0 branch)
            const int sep = np, im = i == 0 ? np - 1 : i - 1;
            const int X = i, Y = sep + i, Z = 2 * sep + i;
            out(X) = (at(Z, 0, 0) - at(Z, 0, -1)) / dx - (at(Y, 0, 0) - at(sep + im, 0, 0)) / dx_fine;
            out(Y) = (at(X, 0, 0) - at(im, 0, 0)) / dx_fine - (at(Z, 0, 0) - at(Z, -1, 0)) / dx;
            if (i > 0) out(Z) = (at(Y, 0, 0) - at(Y, -1, 0) - at(X, 0, 0) + at(X, 0, -1)) * fac;
            else out(Z) = (at(Y, 0, 0) - at(Y, -1, 0)) / dx - (at(X, 0, 0) - at(X, 0, -1)) / dx;
        }
        else if (OP == 1 || OP == 2)
        {
            if (OP == 1)
            {
                out(0) = 0.0;
                out(1) = 0.0;
            }
            else
            {
                out(0) = (bt(0, 0, 0) - bt(0, 0, -1)) * fac;
                out(1) = (-bt(0, 0, 0) + bt(0, -1, 0)) * fac;
            }
            out(2) = (at(1, 0, 0) - at(1, -1, 0) - at(0, 0, 0) + at(0, 0, -1)) * fac;
        }
        else if (OP == 3)
        {
            const double f = fac * scale;
            out(0) = (-at(2, 0, 0) + at(2, 0, 1)) * f;
            out(1) = (at(2, 0, 0) - at(2, 1, 0)) * f;
            Ef[p] = (-at(1, 0, 0) + at(1, 1, 0) + at(0, 0, 0) - at(0, 0, 1)) * f;
            out(0) += at(1, 0, 0) * c * scale;
            out(1) -= at(0, 0, 0) * c * scale;
        }
        else if (OP == 4)
        {
            out(0) = 0.25 * (-bt(2, 0, 0) * (at(1, 0, 0) + at(1, -1, 0)) - bt(2, 0, 1) * (at(1, 0, 1) + at(1, -1, 1)));
            out(1) = 0.25 * (bt(2, 0, 0) * (at(0, 0, 0) + at(0, 0, -1)) + bt(2, 1, 0) * (at(0, 1, 0) + at(0, 1, -1)));
            Ef[p] = 0.5 * (bt(0, 0, 0) * at(1, 0, 0) + bt(0, 0, 1) * at(1, 0, 1) - bt(1, 0, 0) * at(0, 0, 0) -
                           bt(1, 1, 0) * at(0, 1, 0));
        }
        else
        {
            const double f = fac * scale;
            out(0) = (-at(0, 0, 0) + at(0, 0, 1)) * f;
            out(1) = (-at(0, 1, 0) + at(0, 0, 0)) * f;
        }
    }
}

int trapezoid_points(double c)
{
    int n = 64;
    while (n < (1 << 20) && c * n < 48.0) n *= 2;
    return n;
}

// Gauss-Legendre nodes and weights on [0, pi]: the roots of P_N by Newton's
// method from the Chebyshev-like first guesses cos(pi (i + 3/4) / (N + 1/2)),
// P_N and P_N' from the three-term recurrence; weights 2 / ((1 - t^2) P_N'^2)
void gauss_legendre_0_pi(int N, std::vector<double>& x, std::vector<double>& w)
{
    x.assign(N, 0.0);
    w.assign(N, 0.0);
    for (int i = 0; i < (N + 1) / 2; ++i)
    {
        double t = std::cos(M_PI * (i + 0.75) / (N + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it)
        {
            double p0 = 1.0, p1 = t;
            for (int k = 2; k <= N; ++k)
            {
                const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = N * (t * p1 - p0) / (t * t - 1.0);
            const double dt = p1 / dp;
            t -= dt;
            if (std::fabs(dt) < 1e-16) break;
        }
        const double wt = 2.0 / ((1.0 - t * t) * dp * dp);
        // t and -t, mapped from [-1, 1] to [0, pi]
        x[i] = 0.5 * M_PI * (1.0 - t);
        x[N - 1 - i] = 0.5 * M_PI * (1.0 + t);
        w[i] = w[N - 1 - i] = 0.5 * M_PI * wt;
    }
}
}  // namespace

// origin_val (helmholtz_lookup.hpp:94-119): the Gauss hypergeometric series
// 2F1(1/2, 1/2; 1; z) summed until a term falls below 1e-20
double helm2d_origin(double c)
{
    const double z = (2.0 / (2.0 + c * c / 2.0)) * (2.0 / (2.0 + c * c / 2.0));
    double a = 0.5, b = 0.5, cc = 1.0, term = a * b * z / cc, value = 1.0 + term;
    for (int n = 1; std::fabs(term) > 1e-20 && n < 100000000;)
    {
        a += 1.0, b += 1.0, cc += 1.0, ++n;
        term *= a * b * z / cc / n;
        value += term;
    }
    return 0.5 / (2.0 + c * c / 2.0) * value;
}

namespace
{
// get(n, m) for a table (nm null: 0 <= n < nx, 0 <= m < ny) or for the nx
// offsets of nm (ny = 1); extent = the largest |offset| + 1 on either axis
void launch_lgf(Ctx& c, double cz, int nx, int ny, const int* dev_nm, int extent, double* dev_out)
{
    const int total = nx * ny;
    if (cz > 0.0)
        helm2d_table_kernel<<<(total + 127) / 128, 128, 0, c.stream>>>(nx, ny, dev_nm, cz, trapezoid_points(cz),
                                                                       dev_out);
    else
    {
        // node count grows with the offsets (the integrand varies on a scale 1 / |n| near 0)
        const int npts = std::min(8192, 96 + 6 * extent);
        std::vector<double> x, w;
        gauss_legendre_0_pi(npts, x, w);
        x.insert(x.end(), w.begin(), w.end());
        DevBuf<double> d;
        d.upload(x, c.stream);
        lap2d_table_kernel<<<(total + 127) / 128, 128, 0, c.stream>>>(nx, ny, dev_nm, d.p, d.p + npts, npts, dev_out);
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));  // the nodes are freed on return
    }
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}
}  // namespace

void helm2d_check_table(double cz, int nx, int ny)
{
    if (!(cz >= 0.0) || nx < 1 || ny < 1) throw Error(IBLGF_EINVAL, "need c >= 0 and a non-empty table");
    if ((long long)nx * ny > (1ll << 28)) throw Error(IBLGF_EINVAL, "the table holds at most 2^28 entries");
}

void helm2d_table(Ctx& c, double cz, int nx, int ny, double* dev_out)
{
    helm2d_check_table(cz, nx, ny);
    launch_lgf(c, cz, nx, ny, nullptr, std::max(nx, ny), dev_out);
}

void helm2d_points(Ctx& c, double cz, int count, const int* host_nm, double* host_out)
{
    if (!(cz >= 0.0) || count < 0 || (count && (!host_nm || !host_out)))
        throw Error(IBLGF_EINVAL, "need c >= 0 and offset / output arrays");
    if (!count) return;
    int extent = 1;
    for (int i = 0; i < 2 * count; ++i)
    {
        if (host_nm[i] == INT_MIN) throw Error(IBLGF_EINVAL, "offset out of range");
        extent = std::max(extent, std::abs(host_nm[i]) + 1);
    }
    DevBuf<int> nm;
    nm.upload(std::vector<int>(host_nm, host_nm + 2 * count), c.stream);
    DevBuf<double> out;
    out.alloc((size_t)count);
    launch_lgf(c, cz, count, 1, nm.p, extent, out.p);
    IBLGF_CUDA(cudaMemcpyAsync(host_out, out.p, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
}

// Blocks are nb x nb with nb <= 4096, and one launch indexes at most
// 2^31 - 1 (unit, node) pairs.
void check_block_extent(int nb, long long units)
{
    if (nb < 3 || nb > 4096) throw Error(IBLGF_EINVAL, "block extent outside 3 .. 4096");
    if (units * nb * nb > 0x7fffffffll) throw Error(IBLGF_EINVAL, "too many (plane, node) pairs per block");
}

UnitMask unit_mask(int n_units, const unsigned char* host_mask)
{
    if (n_units < 1 || n_units > UnitMask::kMax)
        throw Error(IBLGF_EINVAL, "the mode (or plane) count is outside 1 .. 2048");
    UnitMask m{};
    for (int i = 0; i < n_units; ++i)
        if (!host_mask || host_mask[i]) m.w[i >> 5] |= 1u << (i & 31);
    return m;
}

void helm2d_op(Ctx& c, int op, int nb, int n_blocks, int n_modes, double dx, double lz, double scale,
               const unsigned char* host_mode_mask, const double* dev_src, double* dev_dst)
{
    if (op < 0 || op > 4 || nb < 3 || n_blocks < 0 || n_modes < 1 || !(dx > 0.0) || !(lz > 0.0))
        throw Error(IBLGF_EINVAL, "bad Helmholtz operator arguments");
    check_block_extent(nb, 6ll * n_modes);  // components per block of the widest field
    const UnitMask mask = unit_mask(n_modes, host_mode_mask);
    if (!n_blocks) return;
    const int sep = 2 * n_modes;
    const int in_comp = (op == 0 || op == 1) ? sep : 3 * sep;
    const int out_comp = (op == 0 || op == 2) ? sep : 3 * sep;
    auto go = [&](auto kfn) {
        kfn<<<n_blocks, 256, 0, c.stream>>>(nb, n_modes, in_comp, out_comp, dx, lz, scale, mask, dev_src, dev_dst);
    };
    switch (op)
    {
        case 0: go(helm_op_kernel<0>); break;
        case 1: go(helm_op_kernel<1>); break;
        case 2: go(helm_op_kernel<2>); break;
        case 3: go(helm_op_kernel<3>); break;
        default: go(helm_op_kernel<4>); break;
    }
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void helm2d_nonlinear(Ctx& c, int nb, int n_blocks, int n_planes, const unsigned char* host_plane_mask,
                      const double* dev_face, const double* dev_edge, double* dev_dst)
{
    if (nb < 3 || n_blocks < 0) throw Error(IBLGF_EINVAL, "bad nonlinear term arguments");
    check_block_extent(nb, 3ll * n_planes);
    const UnitMask mask = unit_mask(n_planes, host_plane_mask);
    if (!n_blocks) return;
    helm_nonlinear_kernel<<<n_blocks, 256, 0, c.stream>>>(nb, n_planes, mask, dev_face, dev_edge, dev_dst);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void helm2d_real_op(Ctx& c, int op, int nb, int n_blocks, int np, double dx, double dx_fine, double cz, double scale,
                    const double* a, int a_comp, const double* b, int b_comp, double* d, int d_comp, double* e)
{
    // components each operator reads or writes: a, b (0: unused), d, e (0/1)
    static const int need[6][4] = {{3, 0, 3, 0}, {2, 0, 3, 0}, {2, 1, 3, 0}, {3, 0, 2, 1}, {2, 3, 2, 1}, {1, 0, 2, 0}};
    if (op < 0 || op > 5 || nb < 3 || n_blocks < 0 || !(dx > 0.0) || (op == 0 && !(dx_fine > 0.0)))
        throw Error(IBLGF_EINVAL, "bad Helmholtz real operator arguments");
    if (op == 0 && (np < 1 || np > (1 << 20))) throw Error(IBLGF_EINVAL, "bad z plane count");
    check_block_extent(nb, op == 0 ? 3ll * np : 3ll);
    const int m = op == 0 ? np : 1;
    const int* k = need[op];
    if (a_comp < k[0] * m || d_comp < k[2] * m || (k[1] && b_comp < k[1]))
        throw Error(IBLGF_EINVAL, "too few components for the operator");
    if (!n_blocks) return;
    if (!a || !d || (k[1] && !b) || (k[3] && !e)) throw Error(IBLGF_EINVAL, "null field");
    auto go = [&](auto kfn) {
        kfn<<<n_blocks, 256, 0, c.stream>>>(nb, np, dx, dx_fine, cz, scale, a, a_comp, k[1] ? b : nullptr,
                                            k[1] ? b_comp : 0, d, d_comp, k[3] ? e : nullptr);
    };
    switch (op)
    {
        case 0: go(helm_real_op_kernel<0>); break;
        case 1: go(helm_real_op_kernel<1>); break;
        case 2: go(helm_real_op_kernel<2>); break;
        case 3: go(helm_real_op_kernel<3>); break;
        case 4: go(helm_real_op_kernel<4>); break;
        default: go(helm_real_op_kernel<5>); break;
    }
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
}

void helm2d_apply(Ctx& c, double cz, int nx, int ny, const double* dev_f, double* dev_u, double scale)
{
    if (nx > 6144) throw Error(IBLGF_EINVAL, "the uniform 2-D solve takes at most 6144 cells along x");
    if (ny > 65535) throw Error(IBLGF_EINVAL, "the uniform 2-D solve takes at most 65535 cells along y");
    helm2d_check_table(cz, nx, ny);
    DevBuf<double> table;
    table.alloc((size_t)nx * ny);
    helm2d_table(c, cz, nx, ny, table.p);
    const int bx = 128;
    helm2d_apply_kernel<<<dim3((nx + bx - 1) / bx, ny), bx, nx * sizeof(double), c.stream>>>(nx, ny, table.p, dev_f,
                                                                                         dev_u, scale);
    c.launches += 1;
    IBLGF_CUDA(cudaGetLastError());
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));  // the table is freed on return
}
}  // namespace iblgf_b200
