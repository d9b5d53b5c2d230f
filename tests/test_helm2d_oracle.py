"""The 2-D Helmholtz LGF oracle (restating helmholtz_lookup.hpp /
helmholtz.hpp) pinned to the mathematics, since the reference stores no
values of it: get(n, m) = G_c(n, m) - origin_val(c) is the decaying solution
of the five-point screened Poisson equation (Delta_h - c^2) g = delta, and
origin_val(c) (the hypergeometric series) equals the quadrature of
1 / (K - 1/K) / (2 pi). No GPU."""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import helm2d as H  # noqa: E402


@pytest.mark.parametrize("c", [0.1, 0.5, 2.0])
def test_origin_is_the_centre_integral(c):
    npts = 1 << 14
    x = -math.pi + 2 * math.pi * np.arange(npts) / npts
    a = 4 - 2 * np.cos(x) + c * c
    K = 0.5 * (a + np.sqrt(a * a - 4))
    c0 = float((1 / (K - 1 / K)).sum() / npts)
    # the series sums thousands of terms when z is close to 1 (small c)
    assert abs(H.origin_val(c) - c0) < 1e-13 * c0


@pytest.mark.parametrize("c", [0.1, 0.5, 2.0])
def test_lgf_solves_the_screened_poisson_equation(c):
    n = 9
    g = np.zeros((2 * n + 1, 2 * n + 1))
    for i in range(-n, n + 1):
        for j in range(-n, n + 1):
            g[j + n, i + n] = H.lgf(i, j, c)
    r = H.residual(g, c)
    delta = np.zeros_like(r)
    delta[n - 1, n - 1] = 1.0
    assert np.abs(r - delta).max() < 1e-12
    assert np.allclose(g, g.T) and np.allclose(g, g[::-1, :])


def test_mode0_kernel_is_the_laplace_lgf():
    """c = 0: the regularised 2-D LGF (G0(0, 0) = 0, Delta_h G0 = delta),
    equal to the reference's far-field expansion (its table is not in the
    reference tree) to the expansion's own error, O(r^-4)."""
    n = 6
    g = np.array([[H.lap_lgf(i, j) for i in range(-n, n + 1)] for j in range(-n, n + 1)])
    r = H.residual(g, 0.0)
    delta = np.zeros_like(r)
    delta[n - 1, n - 1] = 1.0
    assert abs(g[n, n]) == 0.0 and np.abs(r - delta).max() < 1e-13
    assert abs(H.lap_lgf(1, 0) - 0.25) < 1e-13  # G0(1, 0) = 1/4 exactly
    for (a, b) in [(30, 0), (40, 17), (60, 60), (100, 3)]:
        # the expansion stops at r^-2: its remainder is O(r^-4)
        assert abs(H.lap_lgf(a, b) - H.lap_asym(a, b)) < 0.05 / (a * a + b * b) ** 2


def test_apply_solves_the_equation_on_its_support():
    c = 0.7
    rng = np.random.default_rng(3)
    f = rng.standard_normal((10, 12))
    u = H.apply(c, f)
    # the unbounded solution: (Delta_h - c^2) u = f at every interior cell
    assert np.abs(H.residual(u, c) - f[1:-1, 1:-1]).max() < 1e-11 * np.abs(f).max()


def test_complex_helmholtz_operators_are_mimetic():
    """The restated complex (Fourier-in-z) operators keep the staggered
    identities: div grad = laplace, curl grad = 0, div curl^T = 0, per mode
    (the z derivative of mode i is i omega_i)."""
    rng = np.random.default_rng(1)
    nm, nb, dx, lz = 3, 12, 0.3, 2.0
    sep = 2 * nm
    u = rng.standard_normal((2, sep, nb, nb))
    g = H.helm_op("gradient", u, np.zeros((2, 3 * sep, nb, nb)), nm, dx, lz)
    d = H.helm_op("divergence", g, np.zeros((2, sep, nb, nb)), nm, dx, lz)
    lap = H.helm_op("laplace", u, np.zeros((2, sep, nb, nb)), nm, dx, lz)
    tol = 1e-12 * np.abs(lap).max()
    assert np.abs(d - lap)[:, :, 1:nb - 2, 1:nb - 2].max() < tol
    c = H.helm_op("curl", g, np.zeros((2, 3 * sep, nb, nb)), nm, dx, lz)
    assert np.abs(c)[:, :, 2:nb - 1, 2:nb - 1].max() < tol
    e = rng.standard_normal((2, 3 * sep, nb, nb))
    ct = H.helm_op("curl_transpose", e, np.zeros((2, 3 * sep, nb, nb)), nm, dx, lz, 0.7)
    dd = H.helm_op("divergence", ct, np.zeros((2, sep, nb, nb)), nm, dx, lz)
    assert np.abs(dd)[:, :, 1:nb - 2, 1:nb - 2].max() < tol


def test_nonlinear_term_is_the_cross_product_for_uniform_fields():
    """nonlinear_helmholtz's staggered averages reduce to w x u when the
    fields are uniform on each plane; only the selected planes are written."""
    rng = np.random.default_rng(4)
    npl, nb = 5, 8
    uv = rng.standard_normal((3, npl))
    wv = rng.standard_normal((3, npl))
    face = np.repeat(np.repeat(uv.reshape(1, 3 * npl, 1, 1), nb, 2), nb, 3)
    edge = np.repeat(np.repeat(wv.reshape(1, 3 * npl, 1, 1), nb, 2), nb, 3)
    dst = np.full((1, 3 * npl, nb, nb), 7.0)
    H.nonlinear(face, edge, dst, npl, planes=[1, 3])
    cross = np.cross(wv.T, uv.T).T  # (w x u) per plane
    for i in range(npl):
        for g in range(3):
            block = dst[0, g * npl + i, 1:-1, 1:-1]
            if i in (1, 3):
                assert np.abs(block - cross[g, i]).max() < 1e-14
            else:
                assert (block == 7.0).all()
    assert (dst[0, :, 0, :] == 7.0).all()


def test_mode_selections_follow_the_reference_forms():
    import fourier_z
    assert list(fourier_z.refined_modes(8, 2)) == [0, 1]
    with pytest.raises(ValueError):
        fourier_z.refined_modes(6, 2)  # the reference throws when 2^r does not divide N_modes
    assert list(fourier_z.one_mode_planes(2, 3)) == [6, 7, 8]
    assert list(fourier_z.refined_planes(12, 2)) == [0, 4, 8]


def test_real_operators_agree_with_the_complex_and_plane_forms():
    """The real-valued restatements against the ones pinned above:
    curl_helmholtz_real with Uz is the complex curl of mode 0 (real parts);
    curl_transpose_helmholtz_complex_linear at c = 0 is mode 0's complex
    curl_transpose; curl_helmholtz on fields constant along z is the in-plane
    curl of every plane; nonlinear_linear_helm is the plane convective term
    with u_z = 0; the 2-D curl_transpose is divergence-free."""
    rng = np.random.default_rng(9)
    nb, nblk, dx = 10, 2, 0.4
    I = slice(1, nb - 1)
    # complex layout, one mode: x_re, x_im, y_re, y_im, z_re, z_im
    fc = rng.standard_normal((nblk, 6, nb, nb))
    cc = H.helm_op("curl", fc, np.zeros((nblk, 6, nb, nb)), 1, dx, 1.0)
    r = H.real_op("curl_real_uz", fc[:, [0, 2]], np.zeros((nblk, 3, nb, nb)), b=fc[:, [4]], dx=dx)
    assert np.abs(r[:, :, I, I] - cc[:, [0, 2, 4]][:, :, I, I]).max() < 1e-12
    r0 = H.real_op("curl_real", fc[:, [0, 2]], np.ones((nblk, 3, nb, nb)), dx=dx)
    assert (r0[:, :2, I, I] == 0).all() and np.array_equal(r0[:, 2, I, I], r[:, 2, I, I])
    ct = H.helm_op("curl_transpose", fc, np.zeros((nblk, 6, nb, nb)), 1, dx, 1.0, 0.6)
    d = np.zeros((nblk, 2, nb, nb))
    e = np.zeros((nblk, 1, nb, nb))
    H.real_op("curl_transpose_linear", fc[:, [0, 2, 4]], d, e=e, dx=dx, c=0.0, scale=0.6)
    assert np.abs(d[:, :, I, I] - ct[:, [0, 2]][:, :, I, I]).max() < 1e-12
    assert np.abs(e[:, 0, I, I] - ct[:, 4, I, I]).max() < 1e-12
    # planes: the same 2-D field on every plane -> no z differences
    npl = 4
    f2 = rng.standard_normal((nblk, 3, nb, nb))
    planes = np.repeat(f2, npl, axis=1)  # groups x, y, z of npl planes each
    cp = H.real_op("curl_planes", planes, np.zeros((nblk, 3 * npl, nb, nb)), n_planes=npl, dx=dx, dx_fine=0.1)
    ref = H.real_op("curl_real_uz", f2[:, :2], np.zeros((nblk, 3, nb, nb)), b=f2[:, [2]], dx=dx)
    for i in range(npl):
        got = cp[:, [i, npl + i, 2 * npl + i]]
        assert np.abs(got[:, :, I, I] - ref[:, :, I, I]).max() < 1e-12
    # linearised convective term = the plane form with u_z = 0
    u = rng.standard_normal((nblk, 3, nb, nb))
    u[:, 2] = 0.0
    w = rng.standard_normal((nblk, 3, nb, nb))
    full = H.nonlinear(u, w, np.zeros((nblk, 3, nb, nb)), 1)
    d = np.zeros((nblk, 2, nb, nb))
    e = np.zeros((nblk, 1, nb, nb))
    H.real_op("nonlinear_linear", u[:, :2], d, b=w, e=e)
    assert np.abs(d[:, :, I, I] - full[:, :2, I, I]).max() < 1e-13
    assert np.abs(e[:, 0, I, I] - full[:, 2, I, I]).max() < 1e-13
    s = rng.standard_normal((nblk, 1, nb, nb))
    f = H.real_op("curl_transpose_2d", s, np.zeros((nblk, 2, nb, nb)), dx=dx, scale=0.5)
    div = f[:, 0, 1:-2, 2:-1] - f[:, 0, 1:-2, 1:-2] + f[:, 1, 2:-1, 1:-2] - f[:, 1, 1:-2, 1:-2]
    assert np.abs(div[:, 1:, 1:]).max() < 1e-12


def test_mode_and_plane_masks_are_bytes_per_unit():
    """The host side of the mode / plane selections: indices or a boolean
    sequence become one byte per unit; out-of-range indices and wrong-length
    boolean masks are refused before the library is called."""
    import iblgf_b200 as B
    assert B.Solver._unit_mask(4, None) is None
    assert B.Solver._unit_mask(4, [2]).tolist() == [0, 0, 1, 0]
    assert B.Solver._unit_mask(4, range(2)).tolist() == [1, 1, 0, 0]
    assert B.Solver._unit_mask(4, np.array([True, False, False, True])).tolist() == [1, 0, 0, 1]
    assert B.Solver._unit_mask(3, []).tolist() == [0, 0, 0]
    for bad in ([4], [-1], np.array([True, False])):
        with pytest.raises(B.IblgfError):
            B.Solver._unit_mask(4, bad)


@pytest.mark.parametrize("c", [0.5, 1.2])
def test_lgf_matches_a_direct_solve_of_the_lattice_equation(c):
    """Independent of the quadrature: (Delta_h - c^2) g = delta solved as a
    sparse linear system on [-L, L]^2 with g = 0 outside (the kernel decays
    like e^{-c r}, so L = 90 leaves < 1e-15 of the kernel at the edge)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    L = 90
    n = 2 * L + 1
    one = np.ones(n)
    d2 = sp.diags([one[:-1], -2 * one, one[:-1]], [-1, 0, 1])
    eye = sp.identity(n)
    A = (sp.kron(eye, d2) + sp.kron(d2, eye) - c * c * sp.identity(n * n)).tocsc()
    rhs = np.zeros(n * n)
    rhs[L * n + L] = 1.0
    g = spl.spsolve(A, rhs).reshape(n, n)
    for (a, b) in [(0, 0), (1, 0), (3, 2), (7, 1), (12, 9)]:
        assert abs(g[L + b, L + a] - H.lgf(a, b, c)) < 1e-13 * abs(g[L, L])


def test_unknown_operator_names_are_refused():
    """Checked before any tensor or device is touched (a stand-in for the
    solver carries only the operator tables)."""
    import types

    import iblgf_b200 as B
    stub = types.SimpleNamespace(HELM_OPS=B.Solver.HELM_OPS, HELM_REAL_OPS=B.Solver.HELM_REAL_OPS)
    with pytest.raises(B.IblgfError):
        B.Solver.helm2d_op(stub, "grad", None, None, 1, 1.0, 1.0)
    with pytest.raises(B.IblgfError):
        B.Solver.helm2d_real_op(stub, "curl_helmholtz", None, None)
