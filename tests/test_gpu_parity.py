"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances: FP64 plain path <= 1e-12 relative L-inf (the FP64 parity bar);
FP32 FFT/MAC path <= 1e-5 relative L-inf; integer data (keys, lists, masks)
bit-exact.
"""
import json
import os
import sys

import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(case, precision=B.FP64, **kw):
    n_levels = getattr(case, "n_levels", 0)
    pred = getattr(case, "predicate", None)
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=n_levels, predicate=pred)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=n_levels, predicate=pred, precision=precision, **kw)
    return o, g


def test_lgf_table_on_device():
    g = B.Solver((-24,) * 3, (48,) * 3, 6, 1.0, [((-24,) * 3, (48,) * 3)])
    tab = g.lgf_table()
    gold = json.load(open(os.path.join(HERE, "golden", "lgf_table_sample.json")))["entries"]
    idx = [(a * (2 + 3 * a + a * a)) // 6 + b * (b + 1) // 2 + c for a, b, c, _ in gold]
    ref = np.array([v for *_, v in gold])
    assert np.max(np.abs(tab[idx] - ref) / ref) < 5e-14
    rng = np.random.default_rng(1)
    xyz = rng.integers(-160, 160, size=(4000, 3))
    xyz[:500] = rng.integers(-8, 8, size=(500, 3))
    ref = np.array([O.lgf_get(*p) for p in xyz])
    assert np.max(np.abs(g.lgf_get(xyz) - ref) / np.abs(ref)) < 1e-13


@pytest.mark.parametrize("name", ["ffm", "vr0", "vr1", "uniform_64", "amr_small"])
def test_domain_lists_masks_bit_identical(name):
    case = {"ffm": lambda: S.ImpulseFmm(), "vr0": lambda: S.VortexRingPoisson(0),
            "vr1": lambda: S.VortexRingPoisson(1), "uniform_64": lambda: S.GaussianPoisson("uniform_64"),
            "amr_small": lambda: S.GaussianPoisson("amr_small")}[name]()
    o, g = pair(case)
    assert (o.n, o.base_level, o.depth) == (g.n, g.base_level, g.depth)
    assert np.array_equal(o.keys, g.keys) and np.array_equal(o.levels, g.levels)
    assert np.array_equal(o.flags, g.flags) and np.array_equal(o.bbase, g.bbase)
    for a, b in zip(o.lists(), g.lists()):
        assert np.array_equal(a, b)
    for idx in [0] + [15 + 2 * r + n for r in range(g.depth - g.base_level) for n in (0, 1)]:
        assert np.array_equal(o.masks(idx), g.masks(idx)), idx


def _conv_kats(precision, tol):
    torch = pytest.importorskip("torch")
    for N, kind in ((8, "fft"), (16, "delta")):
        P = 2 * N - 1
        g = B.Solver((-4 * N,) * 3, (8 * N,) * 3, N - 2, 1.0, [((-2 * N + 4,) * 3, ((N - 2) * 2,) * 3)],
                     precision=precision)
        if kind == "fft":
            i, j, k = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
            src = np.sin(i) + 0.1 * j - 0.2 * k
            ker = np.zeros((P, P, P))
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        ker[N - 1 + dx, N - 1 + dy, N - 1 + dz] = 0.3 + 0.1 * dx + 0.05 * dy - 0.02 * dz
            ker[N - 1, N - 1, N - 1] = 1.2345
        else:
            src = np.zeros((N, N, N))
            src[N // 3, N // 4, N // 2] = 1.0
            a = np.arange(P) - N + 1
            ker = np.vectorize(O.lgf_get)(a[:, None, None], a[None, :, None], a[None, None, :])
        ref = O.block_conv(src, ker)
        ts = torch.tensor(src.ravel(order="F"), device="cuda", dtype=torch.float64)
        tk = torch.tensor(ker.ravel(order="F"), device="cuda", dtype=torch.float64)
        to = torch.zeros(N ** 3, device="cuda", dtype=torch.float64)
        g.conv_block(ts.data_ptr(), tk.data_ptr(), to.data_ptr(), 1.0)
        out = to.cpu().numpy().reshape((N, N, N), order="F")
        assert rel_linf(out, ref) < tol, (N, kind, rel_linf(out, ref))


def test_conv_block_kats_fp64():
    _conv_kats(B.FP64, 1e-12)


def test_conv_block_kats_fp32():
    _conv_kats(B.FP32, 1e-5)


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_fmm_impulse(precision, tol):
    case = S.ImpulseFmm()
    o, g = pair(case, precision)
    src, i0, sc = case.source(o)
    ref = o.fmm_apply(src, o.zeros(), o.base_level, 1, 1.0, 1)
    fs, ft = g.field(src), g.field()
    g.fmm_apply(fs, ft, g.base_level, 1, 1.0, B.AMR2AMR)
    out = g.download(ft)
    assert rel_linf(out, ref) < tol
    # and against the LGF itself (ffmTest.cpp) on the non-correction leaves
    Nb = g.Nb
    r = np.arange(1, Nb - 1)
    for blk in np.nonzero(g.leaf & ~g.correction)[0][:40]:
        b = g.bbase[blk]
        ex = np.vectorize(O.lgf_get)(b[0] + r[None, None, :] - 1 - sc[0], b[1] + r[None, :, None] - 1 - sc[1],
                                     b[2] + r[:, None, None] - 1 - sc[2])
        assert np.abs(out[blk, 1:-1, 1:-1, 1:-1] - ex).max() < 5e-8 + tol


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3])
@pytest.mark.parametrize("nlas", [0, 1])
@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_fmm_apply_random_amr(nlas, precision, tol, variant):
    """Every sibling-group MAC variant (0, 1: direct kernel tile shapes; 2:
    block-Toeplitz; 3: tensor cores; 2 and 3 are FP32 only, the FP64 path
    runs variant 0 instead; -1: the autotuner's choice) against the oracle."""
    case = S.GaussianPoisson("amr_small")
    o, g = pair(case, precision)
    g.mac_variant(variant)
    rng = np.random.default_rng(7)
    src = rng.standard_normal((o.n, o.Nb, o.Nb, o.Nb))
    tgt0 = rng.standard_normal((o.n, o.Nb, o.Nb, o.Nb))
    fs, ft = g.field(src), g.field(tgt0)
    for level in range(o.base_level, o.depth):
        ref = o.fmm_apply(src, tgt0, level, nlas, 0.75, 1)
        g.upload(ft, tgt0)
        g.fmm_apply(fs, ft, level, nlas, 0.75, B.AMR2AMR)
        out = g.download(ft)
        assert rel_linf(out - tgt0, ref - tgt0) < tol, (level, rel_linf(out - tgt0, ref - tgt0))
    if variant < 0:
        rec = g.mac_tuning()
        assert rec and all(r["choice"] in (0, 1, 2, 3) for r in rec)
        assert all((r["ms"][2] is None) == (precision == B.FP64) for r in rec)
        assert all((r["ms"][3] is None) == (precision == B.FP64) for r in rec)


@pytest.mark.parametrize("n_levels", [0, 1])
def test_poisson_vortex_ring(n_levels):
    case = S.VortexRingPoisson(n_levels)
    o, g = pair(case)
    src, ex = case.fields(o)
    ref = o.apply_lgf(src)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    out = g.download(ft)
    assert rel_linf(out, ref) < 1e-12
    assert case.finest_linf(g, out, ex) < case.exp_linf


@pytest.mark.parametrize("name", ["uniform_small", "amr_small", "uniform_64"])
@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_poisson_gaussian(name, precision, tol):
    case = S.GaussianPoisson(name)
    o, g = pair(case, precision)
    src = case.fields(o)
    ref = o.apply_lgf(src)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    out = g.download(ft)
    assert rel_linf(out, ref) < tol
    # a second solve on the same context (cached plans and spectra) is identical
    g.zero(ft)
    g.apply_lgf(fs, ft)
    assert np.array_equal(g.download(ft), out)


def test_capi_errors_are_status_codes():
    g = B.Solver((-24,) * 3, (48,) * 3, 6, 1.0, [((-24,) * 3, (48,) * 3)])
    with pytest.raises(B.IblgfError):
        g.fmm_apply(0, 99, g.base_level, 1)
    with pytest.raises(B.IblgfError):
        g.fmm_apply(0, 0, g.depth + 3, 1)
    with pytest.raises(B.IblgfError):
        g.upload(0, np.zeros(5))


@pytest.mark.parametrize("name", ["vr1", "amr_small"])
def test_domain_import_matches(name):
    """iblgf_domain_import (the drop-in path: the reference's Domain builds the
    tree) gives the same octants, lists and masks as building it here."""
    case = {"vr1": lambda: S.VortexRingPoisson(1), "amr_small": lambda: S.GaussianPoisson("amr_small")}[name]()
    o, g = pair(case)
    gi = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                  import_octants=(o.keys[::-1].copy(), o.flags[::-1].copy()))
    assert np.array_equal(gi.keys, o.keys) and np.array_equal(gi.flags, o.flags)
    assert np.array_equal(gi.bbase, o.bbase) and np.array_equal(gi.levels, o.levels)
    for a, b in zip(o.lists(), gi.lists()):
        assert np.array_equal(a, b)
    for idx in [0] + [15 + 2 * r + n for r in range(gi.depth - gi.base_level) for n in (0, 1)]:
        assert np.array_equal(o.masks(idx), gi.masks(idx)), idx


def _run_adapter(tmp_path, case, o, src, mode="poisson", alpha=0.0, level=0):
    import struct
    import subprocess
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("7i", case.block_extent, *case.bd_base, *case.bd_extent))
        f.write(struct.pack("d", case.dx_base))
        f.write(struct.pack("i", o.n))
        f.write(o.keys.astype(np.uint64).tobytes())
        f.write(o.flags.astype(np.int32).tobytes())
        f.write(np.ascontiguousarray(src).tobytes())
    root = os.path.dirname(HERE)
    subprocess.run(["make", "-s", "-C", os.path.join(root, "tests", "cpp")], check=True)
    subprocess.run([os.path.join(root, "tests", "cpp", "adapter_mock"), str(fin), str(fout), mode, repr(alpha),
                    str(level)], check=True)
    return np.fromfile(fout, dtype=np.float64)


def test_cpp_adapter_poisson_solve(tmp_path):
    """The reference-style C++ adapter (PoissonSolver<Setup>::solve<Src,Tgt>)
    over a stand-in domain in shuffled iteration order reproduces the oracle."""
    case = S.GaussianPoisson("amr_small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    src = case.fields(o)
    ref = o.apply_lgf(src)
    out = _run_adapter(tmp_path, case, o, src).reshape(ref.shape)
    # leaves carry the solution (poisson.hpp:761-781); non-leaf targets stay 0
    assert rel_linf(out, ref) < 1e-12


def test_cpp_adapter_integrating_factor_and_kernel_dispatch(tmp_path):
    """Through the C++ adapter: PoissonSolver::apply_lgf_IF (poisson.hpp:428-494),
    Fmm::apply with an LGF_GL kernel (full sweep, non-leaf sources, scale 0.5)
    and with an LGF_GE kernel (neighbour-only branch at alpha_base 4^(level -
    base)), each against the oracle (FP64)."""
    case = S.GaussianPoisson("amr_small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    src = case.fields(o)
    alpha = 0.05
    out = _run_adapter(tmp_path, case, o, src, "if", alpha).reshape(src.shape)
    assert rel_linf(out, o.apply_if(src, alpha)) < 1e-12
    for level in range(o.base_level, o.depth):
        out = _run_adapter(tmp_path, case, o, src, "fmm_gl", 0.0, level).reshape(src.shape)
        assert rel_linf(out, o.fmm_apply(src, o.zeros(), level, 1, 0.5, 1)) < 1e-12
        a = alpha * 4.0 ** (level - o.base_level)
        out = _run_adapter(tmp_path, case, o, src, "fmm_ge", alpha, level).reshape(src.shape)
        ref = o.fmm_apply_ge(src, o.zeros(), level, 0, 1.0, a)
        assert rel_linf(out, ref) < 1e-12, level


def test_cpp_adapter_operators_and_kernel_objects(tmp_path):
    """Operator::levelGradient (gradient, then the target's buffer exchange,
    operators.hpp:588-606) on every level and the per-block
    Operator::curl<face, edge>(it->data(), dx_level) on every octant through
    the adapter, against the oracle; LGF_GL::get, LGF_GE::get and
    Helmholtz<2>::get at fixed offsets against the oracle's kernels."""
    case = S.GaussianPoisson("amr_small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    src = case.fields(o)
    out = _run_adapter(tmp_path, case, o, src, "ops").reshape((6,) + src.shape)
    face = [o.zeros() for _ in range(3)]
    for lv in range(o.base_level, o.depth):
        g = o.op(1, [src], [o.zeros() for _ in range(3)], lv, 1.0)
        for k in range(3):
            on_level = o.levels == lv
            face[k][on_level] = o.buffer_exchange(g[k], lv)[on_level]
    for k in range(3):
        assert rel_linf(out[k], face[k]) < 1e-13, k
    edge = o.op(3, face, [o.zeros() for _ in range(3)], -1, 1.0)
    for k in range(3):
        assert rel_linf(out[3 + k], edge[k]) < 1e-13, k
    alpha = 0.3
    vals = _run_adapter(tmp_path, case, o, src, "kernels", alpha)
    pts = [(i % 7 - 3, (i // 7) % 5 - 2, i // 35 * 37 - 5) for i in range(64)]
    gl = np.array([O.lgf_get(*p) for p in pts])
    ge = np.array([o.lgf_ge_get(*p, alpha) for p in pts])
    assert np.abs(vals[:64] - gl).max() < 1e-13 * np.abs(gl).max()
    assert np.abs(vals[64:128] - ge).max() < 1e-13 * np.abs(ge).max()
    # Helmholtz<2> (c = alpha): get, get after change_level(1) (c / 2), and the
    # default object (c = 0.1, origin 0 until a level or c is set)
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import helm2d as H
    p2 = [(i % 5 - 2, i // 5 * 3 - 4) for i in range(16)]
    for j, c in enumerate((alpha, alpha / 2)):
        ref = np.array([H.lgf(n, m, c) for n, m in p2])
        assert np.abs(vals[128 + 16 * j:144 + 16 * j] - ref).max() < 1e-13 * np.abs(ref).max()
    h0 = H.lgf(3, 1, 0.1) + H.origin_val(0.1)
    assert abs(vals[160] - h0) < 1e-13 * abs(h0) and vals.size == 161


@pytest.mark.parametrize("op,n_in,n_out", [(0, 1, 1), (1, 1, 3), (2, 3, 1), (3, 3, 3), (4, 3, 3), (5, 6, 3)])
def test_mimetic_operators(op, n_in, n_out):
    """Operator::laplace/gradient/divergence/curl/curl_transpose/nonlinear after a
    same-level buffer exchange, every level, against the oracle."""
    case = S.GaussianPoisson("amr_small")
    o, g = pair(case)
    rng = np.random.default_rng(11 + op)
    ins = [rng.standard_normal((o.n, o.Nb, o.Nb, o.Nb)) for _ in range(n_in)]
    outs0 = [rng.standard_normal((o.n, o.Nb, o.Nb, o.Nb)) for _ in range(n_out)]
    # buffers from the exchange on every level, as the level wrappers do
    ref_in = ins
    for lv in range(o.depth):
        ref_in = [o.buffer_exchange(a, lv) for a in ref_in]
    ref = o.op(op, ref_in, outs0, -1, 0.7)
    fi = [g.field(a) for a in ins]
    fo = [g.field(a) for a in outs0]
    for lv in range(g.depth):
        for f in fi:
            g.buffer_exchange(f, lv)
    for f, r in zip(fi, ref_in):
        assert np.array_equal(g.download(f), r)
    g.op(op, fi, fo, -1, 0.7)
    for f, r in zip(fo, ref):
        assert rel_linf(g.download(f), r) < 1e-13


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
@pytest.mark.parametrize("alpha", [0.05, 0.8])
def test_integrating_factor_apply_if(precision, tol, alpha):
    """apply_lgf_IF: LGF_GE neighbour-only FMM per level (alpha x 4^level) with
    the leaf copy, coarsification and correction-buffer interpolation."""
    case = S.GaussianPoisson("amr_small")
    o, g = pair(case, precision)
    src = case.fields(o)
    ref = o.apply_if(src, alpha)
    fs, ft = g.field(src), g.field()
    g.apply_if(fs, ft, alpha)
    assert rel_linf(g.download(ft), ref) < tol


@pytest.mark.parametrize("precision", [B.FP64, B.FP32])
@pytest.mark.parametrize("alpha", [0.0004, 0.002, 0.05])
def test_integrating_factor_direct_sums_match_transforms(precision, alpha):
    """The integrating factor's neighbour sweeps as direct separable sums
    (taken when e^{-2a} I_m(2a) is negligible beyond R = 4, 6 or 8 cells; the
    three alphas cover the three radii on the base level, alpha x 4^level on
    the finer ones) against the same sweeps by block FFT convolution, and
    against the oracle."""
    case = S.GaussianPoisson("amr_small")
    o, g = pair(case, precision)
    src = case.fields(o)
    ref = o.apply_if(src, alpha)
    fs, ft = g.field(src), g.field()
    out = {}
    for direct in (False, True):
        g.ge_direct(direct)
        g.zero(ft)
        n0 = g.launches()
        g.apply_if(fs, ft, alpha)
        out[direct] = (g.download(ft), g.launches() - n0)
    assert out[True][1] < out[False][1]  # fewer launches: the direct path ran
    tol = 1e-13 if precision == B.FP64 else 1e-5
    assert rel_linf(out[True][0], out[False][0]) < tol
    assert rel_linf(out[True][0], ref) < (1e-12 if precision == B.FP64 else 1e-5)


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_poisson_stream_mask(precision, tol):
    """apply_lgf with MASK_TYPE::STREAM (base level only, stream mask: sources
    are the non-correction base blocks) as pad_velocity uses it."""
    case = S.GaussianPoisson("amr_small")
    o, g = pair(case, precision)
    src = case.fields(o)
    ref = o.apply_lgf(src, fmm_type=0)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft, fmm_type=B.STREAM)
    assert rel_linf(g.download(ft), ref) < tol
