"""Test infrastructure: the oracle of the 2-D Helmholtz lattice Green's function
(numpy). Only tests import it; it is never part of the product path.

Restates include/iblgf/lgf/helmholtz_lookup.hpp:
  * integrandFcn / integralHelmholtzTrap (:134-150): the trapezoidal rule on
    [-pi, pi] of (1 - cos(m x) / K^n) / (K - 1/K) / (2 pi), a = 4 - 2 cos x + c^2,
    K = (a + sqrt(a^2 - 4)) / 2, refined (point count doubled) until the
    relative change falls below the tolerance (boost::math::quadrature::
    trapezoidal, tolerance 1e-20 in the reference; here until it stops
    changing in FP64);
  * origin_val / hypergeometric (:94-119): 0.5 / (2 + c^2/2) times the Gauss
    series 2F1(1/2, 1/2; 1; z), z = (2 / (2 + c^2/2))^2, summed until a term
    falls below 1e-20;
and include/iblgf/lgf/helmholtz.hpp:152-163, Helmholtz<2>::get = the integral
at (max(|n|, |m|), min(|n|, |m|)) minus origin_val. For c = 0 (mode 0, LGF_GL<2>,
include/iblgf/lgf/lgf_gl.hpp:93-99, lgf_gl_lookup.hpp:46-60, 121-131) the
regularised 2-D LGF G0(n, m) = 1/pi int_0^pi (1 - e^{-|n| s} cos(m x)) /
(2 sinh s) dx, cosh s = 2 - cos x, by Gauss-Legendre quadrature (numpy), and
the reference's far-field expansion asym() restated for comparison.
"""
import functools
import math

import numpy as np


def origin_val(c):
    z = (2.0 / (2.0 + c * c / 2.0)) ** 2
    a, b, cc = 0.5, 0.5, 1.0
    term = a * b * z / cc
    value = 1.0 + term
    n = 1
    while abs(term) > 1e-20:
        a, b, cc, n = a + 1.0, b + 1.0, cc + 1.0, n + 1
        term *= a * b * z / cc / n
        value += term
    return 0.5 / (2.0 + c * c / 2.0) * value


def integral(n, m, c, tol=1e-16, max_points=1 << 22):
    """integralHelmholtzTrap(n, m, c): trapezoidal rule refined by doubling."""
    def trap(npts):
        x = -math.pi + 2.0 * math.pi * np.arange(npts) / npts
        a = 4.0 - 2.0 * np.cos(x) + c * c
        K = 0.5 * (a + np.sqrt(a * a - 4.0))
        f = (1.0 - np.cos(x * m) / K ** n) * (1.0 / (K - 1.0 / K)) / (2.0 * math.pi)
        return float(f.sum() * (2.0 * math.pi / npts))
    npts = 16
    prev = trap(npts)
    while npts < max_points:
        npts *= 2
        cur = trap(npts)
        if abs(cur - prev) <= tol * abs(cur):
            return cur
        prev = cur
    return prev


@functools.lru_cache(maxsize=64)
def _gauss_legendre_0_pi(npts):
    x, w = np.polynomial.legendre.leggauss(npts)
    x = (x + 1.0) * math.pi / 2.0
    t = 2.0 * np.sin(x / 2.0) ** 2      # 1 - cos x, without cancellation
    r = np.sqrt(t * (2.0 + t))          # sinh s
    return x, w * math.pi / 2.0, np.log1p(t + r), r


def lap_lgf(n, m, npts=None):
    """G0(n, m), the 2-D LGF of the five-point Laplacian with G0(0, 0) = 0
    (node count growing with the offset; numpy's nodes lose accuracy for
    counts in the thousands)."""
    n, m = abs(int(n)), abs(int(m))
    if n < m:
        n, m = m, n
    x, w, s, r = _gauss_legendre_0_pi(npts or 256 + 8 * n)
    return float((w * (1.0 - np.exp(-n * s) * np.cos(m * x)) / (2.0 * r)).sum() / math.pi)


def lap_asym(n1, n2):
    """-LGF_GL_Lookup::asym(n1, n2) (lgf_gl_lookup.hpp:121-131): the
    reference's mode-0 kernel beyond its table."""
    c_fund, integral_val = -0.18124942796, -0.076093998454228
    r = math.sqrt(n1 * n1 + n2 * n2)
    theta = math.atan2(n2, n1)
    return -(-0.5 / math.pi * math.log(r) + c_fund + integral_val + 1.0 / 24.0 / math.pi * math.cos(4 * theta) / r / r)


def lgf(n, m, c):
    """Helmholtz<2>::get at the offset (n, m); c = 0: G0."""
    if c == 0.0:
        return lap_lgf(n, m)
    x, y = abs(int(n)), abs(int(m))
    if x < y:
        x, y = y, x
    return integral(x, y, c) - origin_val(c)


def table(c, nx, ny):
    """get(n, m) for 0 <= n < nx, 0 <= m < ny as an (ny, nx) array."""
    cache = {}
    out = np.zeros((ny, nx))
    for m in range(ny):
        for n in range(nx):
            key = (max(n, m), min(n, m))
            if key not in cache:
                cache[key] = lgf(key[0], key[1], c)
            out[m, n] = cache[key]
    return out


def apply(c, f):
    """u = sum_j get(i - j) f(j) over the uniform grid of f (shape (ny, nx))."""
    ny, nx = f.shape
    t = table(c, nx, ny)
    u = np.zeros_like(f, dtype=np.float64)
    for sy in range(ny):
        for sx in range(nx):
            v = f[sy, sx]
            if v == 0.0:
                continue
            u += v * t[np.abs(np.arange(ny) - sy)][:, np.abs(np.arange(nx) - sx)]
    return u


def residual(g, c):
    """(Delta_h - c^2) applied to g at the interior nodes (five-point)."""
    return (g[1:-1, 2:] + g[1:-1, :-2] + g[2:, 1:-1] + g[:-2, 1:-1] - (4.0 + c * c) * g[1:-1, 1:-1])


# -- complex Helmholtz (Fourier-in-z) block operators on 2-D blocks --------
# include/iblgf/operators/operators.hpp:1516-1545 laplace_helmholtz_complex,
# :1585-1614 gradient_helmholtz_complex, :1763-1795 divergence_helmholtz_complex,
# :1972-2008 curl_helmholtz_complex, :2178-2217 curl_transpose_helmholtz_complex.
# A block holds [component][NB][NB] (x fastest); a scalar field has
# sep = 2 N_modes components (mode i: real 2i, imaginary 2i+1), a vector field
# three groups of sep (x, y, z). Each operator writes the interior nodes
# (1 .. NB-2 on both axes) and reads their one-cell neighbours;
# omega_i = 2 pi i / lz.
def helm_op(op, src, dst, n_modes, dx, lz, scale=1.0, modes=None):
    """op: 'laplace', 'gradient', 'divergence', 'curl', 'curl_transpose';
    src, dst: arrays [n_blocks][ncomp][NB][NB]; dst is updated in place.
    modes: the modes computed (None: all; the _oneMode forms, :1548-1583,
    1620-1652, 1801-1837, 2017-2057, 2224-2270, compute one; the _refined
    forms, :1653-1722, 1839-1887, 2125-2176, the first n_modes / 2^r).
    A mode's components depend on that mode's inputs alone, so a restricted
    form equals the full one on the selected modes' components."""
    if modes is not None:
        out = dst.copy()
        full = helm_op(op, src, dst.copy(), n_modes, dx, lz, scale)
        sep = 2 * n_modes
        groups = 1 if op in ("laplace", "divergence") else 3
        for m in modes:
            for g in range(groups):
                for c in (2 * m, 2 * m + 1):
                    out[:, g * sep + c] = full[:, g * sep + c]
        dst[...] = out
        return dst
    sep = 2 * n_modes
    nb = src.shape[-1]
    I = slice(1, nb - 1)

    def at(c, ox, oy):
        return src[:, c, 1 + oy:nb - 1 + oy, 1 + ox:nb - 1 + ox]

    fac = 1.0 / dx
    om = [2.0 * math.pi * i / lz for i in range(n_modes)]
    if op == "laplace":
        for i in range(sep):
            dst[:, i, I, I] = fac * fac * (-4.0 * at(i, 0, 0) + at(i, 0, -1) + at(i, 0, 1) + at(i, -1, 0) + at(i, 1, 0))
        for i in range(n_modes):
            dst[:, 2 * i, I, I] -= at(2 * i, 0, 0) * om[i] * om[i]
            dst[:, 2 * i + 1, I, I] -= at(2 * i + 1, 0, 0) * om[i] * om[i]
    elif op == "gradient":
        for i in range(sep):
            dst[:, i, I, I] = fac * (at(i, 0, 0) - at(i, -1, 0))
            dst[:, sep + i, I, I] = fac * (at(i, 0, 0) - at(i, 0, -1))
        for i in range(n_modes):
            dst[:, 2 * sep + 2 * i, I, I] = -at(2 * i + 1, 0, 0) * om[i]
            dst[:, 2 * sep + 2 * i + 1, I, I] = at(2 * i, 0, 0) * om[i]
    elif op == "divergence":
        for i in range(sep):
            dst[:, i, I, I] = fac * (-at(i, 0, 0) - at(sep + i, 0, 0) + at(i, 1, 0) + at(sep + i, 0, 1))
        for i in range(n_modes):
            dst[:, 2 * i, I, I] -= at(2 * sep + 2 * i + 1, 0, 0) * om[i]
            dst[:, 2 * i + 1, I, I] += at(2 * sep + 2 * i, 0, 0) * om[i]
    elif op == "curl":
        for i in range(sep):
            dst[:, i, I, I] = fac * (at(2 * sep + i, 0, 0) - at(2 * sep + i, 0, -1))
            dst[:, sep + i, I, I] = fac * (-at(2 * sep + i, 0, 0) + at(2 * sep + i, -1, 0))
            dst[:, 2 * sep + i, I, I] = fac * (at(sep + i, 0, 0) - at(sep + i, -1, 0) - at(i, 0, 0) + at(i, 0, -1))
        for i in range(n_modes):
            dst[:, 2 * i, I, I] += at(sep + 2 * i + 1, 0, 0) * om[i]
            dst[:, 2 * i + 1, I, I] -= at(sep + 2 * i, 0, 0) * om[i]
            dst[:, sep + 2 * i, I, I] -= at(2 * i + 1, 0, 0) * om[i]
            dst[:, sep + 2 * i + 1, I, I] += at(2 * i, 0, 0) * om[i]
    elif op == "curl_transpose":
        f = fac * scale
        for i in range(sep):
            dst[:, i, I, I] = f * (-at(2 * sep + i, 0, 0) + at(2 * sep + i, 0, 1))
            dst[:, sep + i, I, I] = f * (at(2 * sep + i, 0, 0) - at(2 * sep + i, 1, 0))
            dst[:, 2 * sep + i, I, I] = f * (-at(sep + i, 0, 0) + at(sep + i, 1, 0) + at(i, 0, 0) - at(i, 0, 1))
        for i in range(n_modes):
            dst[:, 2 * i, I, I] += at(sep + 2 * i + 1, 0, 0) * om[i] * scale
            dst[:, 2 * i + 1, I, I] -= at(sep + 2 * i, 0, 0) * om[i] * scale
            dst[:, sep + 2 * i, I, I] -= at(2 * i + 1, 0, 0) * om[i] * scale
            dst[:, sep + 2 * i + 1, I, I] += at(2 * i, 0, 0) * om[i] * scale
    else:
        raise ValueError(op)
    return dst


def nonlinear(face, edge, dst, n_planes, planes=None):
    """nonlinear_helmholtz (operators.hpp:2627-2766; _oneMode :2776-2831 and
    _refined :2840-2895 with planes = the planes they compute): face, edge,
    dst are [n_blocks][3 n_planes][NB][NB]; dst's interior nodes of the
    selected planes are overwritten."""
    nb = face.shape[-1]
    I = slice(1, nb - 1)

    def U(c, ox, oy):
        return face[:, c, 1 + oy:nb - 1 + oy, 1 + ox:nb - 1 + ox]

    def W(c, ox, oy):
        return edge[:, c, 1 + oy:nb - 1 + oy, 1 + ox:nb - 1 + ox]

    for i in (range(n_planes) if planes is None else planes):
        x, y, z = i, n_planes + i, 2 * n_planes + i
        dst[:, x, I, I] = (0.5 * W(y, 0, 0) * (U(z, 0, 0) + U(z, -1, 0))
                           - 0.25 * (W(z, 0, 0) * (U(y, 0, 0) + U(y, -1, 0)) + W(z, 0, 1) * (U(y, 0, 1) + U(y, -1, 1))))
        dst[:, y, I, I] = (0.25 * (W(z, 0, 0) * (U(x, 0, 0) + U(x, 0, -1)) + W(z, 1, 0) * (U(x, 1, 0) + U(x, 1, -1)))
                           - 0.5 * W(x, 0, 0) * (U(z, 0, 0) + U(z, 0, -1)))
        dst[:, z, I, I] = 0.5 * (W(x, 0, 0) * U(y, 0, 0) + W(x, 0, 1) * U(y, 0, 1)
                                 - W(y, 0, 0) * U(x, 0, 0) - W(y, 1, 0) * U(x, 1, 0))
    return dst


def real_op(op, a, d, b=None, e=None, n_planes=1, dx=1.0, dx_fine=1.0, c=0.0, scale=1.0):
    """The real-valued family on 2-D blocks ([n_blocks][comp][NB][NB]; d, e
    updated in place at the interior nodes):
    curl_planes        curl_helmholtz, operators.hpp:2305-2414
    curl_real          curl_helmholtz_real, :2059-2081
    curl_real_uz       curl_helmholtz_real with Uz, :2083-2119
    curl_transpose_linear  curl_transpose_helmholtz_complex_linear, :2272-2303
    nonlinear_linear   nonlinear_linear_helm, :2534-2572
    curl_transpose_2d  curl_transpose, two-dimensional branch, :2416-2453"""
    nb = a.shape[-1]
    I = slice(1, nb - 1)

    def A(k, ox, oy):
        return a[:, k, 1 + oy:nb - 1 + oy, 1 + ox:nb - 1 + ox]

    def Bv(k, ox, oy):
        return b[:, k, 1 + oy:nb - 1 + oy, 1 + ox:nb - 1 + ox]

    fac = 1.0 / dx
    if op == "curl_planes":
        sep = n_planes
        for i in range(sep):
            im = sep - 1 if i == 0 else i - 1
            X, Y, Z = i, sep + i, 2 * sep + i
            d[:, X, I, I] = (A(Z, 0, 0) - A(Z, 0, -1)) / dx - (A(Y, 0, 0) - A(sep + im, 0, 0)) / dx_fine
            d[:, Y, I, I] = (A(X, 0, 0) - A(im, 0, 0)) / dx_fine - (A(Z, 0, 0) - A(Z, -1, 0)) / dx
            if i > 0:
                d[:, Z, I, I] = (A(Y, 0, 0) - A(Y, -1, 0) - A(X, 0, 0) + A(X, 0, -1)) * fac
            else:
                d[:, Z, I, I] = (A(Y, 0, 0) - A(Y, -1, 0)) / dx - (A(X, 0, 0) - A(X, 0, -1)) / dx
    elif op in ("curl_real", "curl_real_uz"):
        if op == "curl_real":
            d[:, 0, I, I] = 0.0
            d[:, 1, I, I] = 0.0
        else:
            d[:, 0, I, I] = (Bv(0, 0, 0) - Bv(0, 0, -1)) * fac
            d[:, 1, I, I] = (-Bv(0, 0, 0) + Bv(0, -1, 0)) * fac
        d[:, 2, I, I] = (A(1, 0, 0) - A(1, -1, 0) - A(0, 0, 0) + A(0, 0, -1)) * fac
    elif op == "curl_transpose_linear":
        f = fac * scale
        d[:, 0, I, I] = (-A(2, 0, 0) + A(2, 0, 1)) * f + A(1, 0, 0) * c * scale
        d[:, 1, I, I] = (A(2, 0, 0) - A(2, 1, 0)) * f - A(0, 0, 0) * c * scale
        e[:, 0, I, I] = (-A(1, 0, 0) + A(1, 1, 0) + A(0, 0, 0) - A(0, 0, 1)) * f
    elif op == "nonlinear_linear":
        d[:, 0, I, I] = 0.25 * (-Bv(2, 0, 0) * (A(1, 0, 0) + A(1, -1, 0)) - Bv(2, 0, 1) * (A(1, 0, 1) + A(1, -1, 1)))
        d[:, 1, I, I] = 0.25 * (Bv(2, 0, 0) * (A(0, 0, 0) + A(0, 0, -1)) + Bv(2, 1, 0) * (A(0, 1, 0) + A(0, 1, -1)))
        e[:, 0, I, I] = 0.5 * (Bv(0, 0, 0) * A(1, 0, 0) + Bv(0, 0, 1) * A(1, 0, 1)
                               - Bv(1, 0, 0) * A(0, 0, 0) - Bv(1, 1, 0) * A(0, 1, 0))
    elif op == "curl_transpose_2d":
        f = fac * scale
        d[:, 0, I, I] = (-A(0, 0, 0) + A(0, 0, 1)) * f
        d[:, 1, I, I] = (-A(0, 1, 0) + A(0, 0, 0)) * f
    else:
        raise ValueError(op)
    return d
