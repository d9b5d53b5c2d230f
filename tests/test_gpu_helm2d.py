"""The 2-D Helmholtz lattice Green's function on the device (the kernel of the
reference's Fourier-in-z solvers, lgf::Helmholtz<2>) against the oracle
restating helmholtz_lookup.hpp, and the uniform-grid and Fourier-in-z solves
built on it against the discrete equations they solve."""
import os
import sys

import numpy as np
import pytest

import fourier_z
import iblgf_b200 as B

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import helm2d as H  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    s = B.Solver((-32, -32, -32), (64, 64, 64), 16, 1.0, [((-16, -16, -16), (32, 32, 32))])
    yield s
    s.close()


@pytest.mark.parametrize("c", [0.0, 0.05, 0.3, 1.5])
def test_lgf_table_matches_oracle(g, c):
    t = g.helm2d_lgf(c, 12, 9)
    ref = H.table(c, 12, 9)
    # get(n, m) = G - origin: the reference form cancels digits where G ~ origin
    assert np.abs(t - ref).max() < 1e-13 * np.abs(ref).max()
    if c == 0.0:
        return
    o = np.zeros(1)
    assert abs(B.lib().iblgf_helm2d_origin(c, o.ctypes.data_as(B.ctypes.POINTER(B.ctypes.c_double)))) == 0
    assert abs(o[0] - H.origin_val(c)) < 1e-15 * o[0]


def test_apply_matches_oracle_and_solves_the_equation(g):
    c = 0.7
    rng = np.random.default_rng(11)
    f = rng.standard_normal((10, 12))
    u0 = rng.standard_normal((10, 12))
    u = g.helm2d_apply(c, f, u0, 0.5)
    ref = u0 + 0.5 * H.apply(c, f)
    assert np.abs(u - ref).max() < 1e-12 * np.abs(ref).max()
    w = g.helm2d_apply(c, f)
    assert np.abs(H.residual(w, c) - f[1:-1, 1:-1]).max() < 1e-11 * np.abs(f).max()


def test_mode0_far_field_matches_the_reference_expansion(g):
    """The mode-0 kernel far from the origin against the reference's own
    asym() (lgf_gl_lookup.hpp:121-131), to the expansion's O(r^-4) error."""
    t = g.helm2d_lgf(0.0, 101, 61)
    for (a, b) in [(30, 0), (40, 17), (60, 60), (100, 3)]:
        assert abs(t[b, a] - H.lap_asym(a, b)) < 0.05 / (a * a + b * b) ** 2
        assert abs(t[b, a] - H.lap_lgf(a, b)) < 1e-12  # independent node sets agree to ~1e-13


@pytest.mark.parametrize("z_operator", ["second_order", "spectral"])
def test_fourier_z_solve(g, z_operator):
    """A z-periodic 3-D problem through one 2-D solve per z mode (mode 0 with
    the Laplace kernel): the result satisfies the 3-D equation at every
    interior x-y cell."""
    rng = np.random.default_rng(5)
    nz, ny, nx = 8, 20, 24
    f = rng.standard_normal((nz, ny, nx))
    u = fourier_z.solve(g, f, z_operator)
    lap_xy = u[:, 1:-1, 2:] + u[:, 1:-1, :-2] + u[:, 2:, 1:-1] + u[:, :-2, 1:-1] - 4 * u[:, 1:-1, 1:-1]
    if z_operator == "second_order":
        dzz = np.roll(u, 1, axis=0) + np.roll(u, -1, axis=0) - 2 * u
    else:
        k = fourier_z.mode_wave_numbers(nz, "spectral")
        dzz = np.fft.ifft(-(k ** 2)[:, None, None] * np.fft.fft(u, axis=0), axis=0).real
    r = lap_xy + dzz[:, 1:-1, 1:-1] - f[:, 1:-1, 1:-1]
    assert np.abs(r).max() < 1e-10 * np.abs(f).max()


@pytest.mark.parametrize("op", ["laplace", "gradient", "divergence", "curl", "curl_transpose"])
def test_complex_helmholtz_operators_match_oracle(g, op):
    """The device's complex Helmholtz block operators (2-D blocks, all modes)
    against the restatement of operators.hpp."""
    import torch
    rng = np.random.default_rng(2)
    nm, nb, nblk, dx, lz = 4, 18, 5, 0.25, 1.5
    sep = 2 * nm
    cin = sep if op in ("laplace", "gradient") else 3 * sep
    cout = sep if op in ("laplace", "divergence") else 3 * sep
    src = rng.standard_normal((nblk, cin, nb, nb))
    dst0 = rng.standard_normal((nblk, cout, nb, nb))
    ref = H.helm_op(op, src, dst0.copy(), nm, dx, lz, 0.6)
    s = torch.tensor(src, device="cuda")
    d = torch.tensor(dst0, device="cuda")
    torch.cuda.synchronize()
    g.helm2d_op(op, s, d, nm, dx, lz, 0.6)
    g.synchronize()
    out = d.cpu().numpy()
    assert np.abs(out - ref).max() < 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("sel", ["one_mode", "refined", "bool"])
@pytest.mark.parametrize("op", ["laplace", "gradient", "divergence", "curl", "curl_transpose"])
def test_mode_restricted_operators_match_oracle(g, op, sel):
    """The _oneMode, _refined and ModesBool forms: only the selected modes'
    components change."""
    import torch
    rng = np.random.default_rng(3)
    nm, nb, nblk, dx, lz = 4, 12, 3, 0.5, 2.0
    modes = {"one_mode": [2], "refined": list(fourier_z.refined_modes(nm, 1)),
             "bool": np.array([True, False, False, True])}[sel]
    sep = 2 * nm
    cin = sep if op in ("laplace", "gradient") else 3 * sep
    cout = sep if op in ("laplace", "divergence") else 3 * sep
    src = rng.standard_normal((nblk, cin, nb, nb))
    dst0 = rng.standard_normal((nblk, cout, nb, nb))
    sel_idx = np.flatnonzero(modes) if sel == "bool" else modes
    ref = H.helm_op(op, src, dst0.copy(), nm, dx, lz, 0.4, modes=sel_idx)
    d = torch.tensor(dst0, device="cuda")
    g.helm2d_op(op, torch.tensor(src, device="cuda"), d, nm, dx, lz, 0.4, modes=modes)
    g.synchronize()
    assert np.abs(d.cpu().numpy() - ref).max() < 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("sel", ["all", "one_mode", "refined"])
def test_nonlinear_term_matches_oracle(g, sel):
    import torch
    rng = np.random.default_rng(6)
    npl, nb, nblk = 12, 18, 4
    planes = {"all": None, "one_mode": fourier_z.one_mode_planes(1, 3),
              "refined": fourier_z.refined_planes(npl, 1)}[sel]
    face = rng.standard_normal((nblk, 3 * npl, nb, nb))
    edge = rng.standard_normal((nblk, 3 * npl, nb, nb))
    dst0 = rng.standard_normal((nblk, 3 * npl, nb, nb))
    ref = H.nonlinear(face, edge, dst0.copy(), npl, planes)
    d = torch.tensor(dst0, device="cuda")
    g.helm2d_nonlinear(torch.tensor(face, device="cuda"), torch.tensor(edge, device="cuda"), d, npl,
                       None if planes is None else list(planes))
    g.synchronize()
    assert np.abs(d.cpu().numpy() - ref).max() < 1e-14 * np.abs(ref).max()


def test_unit_masks_are_checked(g):
    import torch
    t = torch.zeros((1, 6, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(B.IblgfError):
        g.helm2d_op("laplace", t, t.clone(), 3, 1.0, 1.0, modes=[3])  # mode index out of range
    with pytest.raises(B.IblgfError):
        big = torch.zeros((1, 3 * 4096, 4, 4), dtype=torch.float64, device="cuda")
        g.helm2d_nonlinear(big, big, big.clone(), 4096)  # more planes than a mask holds


@pytest.mark.parametrize("c", [0.0, 0.3])
def test_point_evaluation_matches_the_table(g, c):
    """iblgf_helm2d_get at scattered signed offsets equals the table entries
    of their absolute values (the kernel is even in both offsets)."""
    rng = np.random.default_rng(8)
    nm = rng.integers(-15, 16, size=(40, 2))
    nm[0] = (15, 0)  # the extent the node count follows, as the table's
    vals = g.helm2d_get(c, nm)
    t = g.helm2d_lgf(c, 16, 16)
    ref = t[np.abs(nm[:, 1]), np.abs(nm[:, 0])]
    assert np.abs(vals - ref).max() < 1e-14 * np.abs(ref).max()
    assert g.helm2d_get(c, np.zeros((0, 2), np.int32)).size == 0


# (a components, b components or 0, d components, e used) per real operator
REAL_SHAPES = {"curl_planes": (15, 0, 15, False), "curl_real": (3, 0, 3, False), "curl_real_uz": (2, 1, 3, False),
               "curl_transpose_linear": (3, 0, 2, True), "nonlinear_linear": (2, 3, 2, True),
               "curl_transpose_2d": (1, 0, 2, False)}


@pytest.mark.parametrize("op", sorted(REAL_SHAPES))
def test_real_operators_match_oracle(g, op):
    """The real-valued family (curl_helmholtz on z planes, curl_helmholtz_real,
    curl_transpose_helmholtz_complex_linear, nonlinear_linear_helm, the 2-D
    curl_transpose) against their restatement; components the operator does
    not write keep their values."""
    import torch
    rng = np.random.default_rng(12)
    na, nbc, nd, use_e = REAL_SHAPES[op]
    nb, nblk, dx, dxf, npl = 12, 3, 0.3, 0.05, 5
    a = rng.standard_normal((nblk, na, nb, nb))
    b = rng.standard_normal((nblk, nbc, nb, nb)) if nbc else None
    d0 = rng.standard_normal((nblk, nd, nb, nb))
    e0 = rng.standard_normal((nblk, 1, nb, nb)) if use_e else None
    kw = dict(n_planes=npl, dx=dx, dx_fine=dxf, c=0.7, scale=1.3)
    d_ref = H.real_op(op, a, d0.copy(), b=b, e=None if e0 is None else e0.copy(), **kw)
    cu = lambda x: None if x is None else torch.tensor(x, device="cuda")
    d, e = cu(d0), cu(e0)
    g.helm2d_real_op(op, cu(a), d, b=cu(b), e=e, n_planes=npl, dx_level=dx, dx_fine=dxf, c=0.7, scale=1.3)
    g.synchronize()
    assert np.abs(d.cpu().numpy() - d_ref).max() < 1e-13 * np.abs(d_ref).max()
    if use_e:
        e_ref = e0.copy()
        H.real_op(op, a, d0.copy(), b=b, e=e_ref, **kw)
        assert np.abs(e.cpu().numpy() - e_ref).max() < 1e-13 * np.abs(e_ref).max()


def test_real_operators_check_their_arguments(g):
    import torch
    t = torch.zeros((2, 2, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(B.IblgfError):
        g.helm2d_real_op("curl_real", t, t.clone())  # the edge output needs 3 components
    with pytest.raises(B.IblgfError):
        g.helm2d_real_op("curl_real_uz", t, torch.zeros((2, 3, 8, 8), dtype=torch.float64, device="cuda"))  # no Uz
    with pytest.raises(B.IblgfError):
        g.helm2d_real_op("curl_planes", torch.zeros((2, 6, 8, 8), dtype=torch.float64, device="cuda"),
                         torch.zeros((2, 6, 8, 8), dtype=torch.float64, device="cuda"), n_planes=3)  # 9 needed


def test_table_and_solve_extents_are_checked(g):
    """Oversized requests are refused before anything is allocated or launched."""
    one = np.zeros(1)
    # 2^29 entries: refused by the library before it allocates or writes
    assert B.lib().iblgf_helm2d_lgf(g.h, 0.5, 1 << 15, 1 << 14, one.ctypes.data_as(B.ctypes.c_void_p)) == B.EINVAL
    with pytest.raises(B.IblgfError):
        g.helm2d_lgf(0.5, 1 << 15, 1 << 14)
    with pytest.raises(B.IblgfError):
        g.helm2d_lgf(-1.0, 4, 4)
    with pytest.raises(B.IblgfError):
        g.helm2d_apply(0.5, np.zeros((4, 6145)))
