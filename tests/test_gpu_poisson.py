"""Leaf-interior field transfers through the C ABI (iblgf_field_upload_leaves /
iblgf_field_download_leaves): the interiors round-trip bit-exact, the upload
zeroes buffers and non-leaf blocks, and apply_lgf on a source uploaded as leaf
interiors gives on every leaf exactly the solution of the same source uploaded
as whole blocks (the solve reads only leaf values: non-leaf sources are
coarsened from the leaves, PoissonSolver::source_coarsify,
poisson.hpp:1136-1194)."""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S

pytestmark = pytest.mark.gpu


def solver(case, precision):
    return B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                    n_levels=getattr(case, "n_levels", 0), predicate=getattr(case, "predicate", None),
                    precision=precision)


def test_leaf_transfers_round_trip():
    g = solver(S.GaussianPoisson("amr_small"), B.FP64)
    rng = np.random.default_rng(3)
    e, leaf = g.block_extent, g.leaf
    assert g.n_leaves == int(leaf.sum()) and 0 < g.n_leaves < g.n
    f = g.field(rng.standard_normal((g.n, g.Nb, g.Nb, g.Nb)))
    vals = rng.standard_normal((g.n_leaves, e, e, e))
    g.upload_leaves(f, vals)
    full = g.download(f)
    np.testing.assert_array_equal(full[leaf][:, 1:-1, 1:-1, 1:-1], vals)
    full[leaf, 1:-1, 1:-1, 1:-1] = 0
    assert not full.any()  # buffers and non-leaf blocks zeroed
    np.testing.assert_array_equal(g.download_leaves(f), vals)
    with pytest.raises(B.IblgfError):
        g.upload_leaves(f, vals[:-1])


@pytest.mark.parametrize("precision", [B.FP64, B.FP32])
def test_solve_from_leaf_upload_matches_block_upload(precision):
    case = S.GaussianPoisson("amr_small")
    g = solver(case, precision)
    src = case.fields(g)
    leaf = g.leaf
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    ref = g.download(ft)[leaf][:, 1:-1, 1:-1, 1:-1]
    g.zero(ft)
    g.upload_leaves(fs, src[leaf][:, 1:-1, 1:-1, 1:-1])
    g.apply_lgf(fs, ft)
    out = g.download_leaves(ft)
    np.testing.assert_array_equal(out, ref)


def test_async_leaf_download_pipeline():
    """Solves of two sources, each solution downloaded asynchronously while
    the next upload and solve run: both equal the synchronous downloads."""
    import torch
    case = S.GaussianPoisson("amr_small")
    g = solver(case, B.FP64)
    e = g.block_extent
    rng = np.random.default_rng(5)
    srcs = [rng.standard_normal((g.n_leaves, e, e, e)) for _ in range(2)]
    fs, ft = g.field(), g.field()
    ref = []
    for x in srcs:
        g.upload_leaves(fs, x)
        g.apply_lgf(fs, ft)
        ref.append(g.download_leaves(ft))
    outs = [torch.empty((g.n_leaves, e, e, e), dtype=torch.float64).pin_memory() for _ in srcs]
    for x, o in zip(srcs, outs):
        g.upload_leaves(fs, x)
        g.apply_lgf(fs, ft)
        g.download_leaves_async(ft, o)
    g.synchronize()
    for r, o in zip(ref, outs):
        np.testing.assert_array_equal(o.numpy(), r)


def test_async_leaf_upload_download_pipeline():
    """Three solves with every input uploaded asynchronously (the next input
    issued right after the current solve, so its copy runs under it) and
    every solution downloaded asynchronously: each equals the synchronous
    solve of that input, bit for bit."""
    import torch
    case = S.GaussianPoisson("amr_small")
    g = solver(case, B.FP32)
    e = g.block_extent
    rng = np.random.default_rng(9)
    srcs = [torch.from_numpy(rng.standard_normal((g.n_leaves, e, e, e))).pin_memory() for _ in range(3)]
    fs, ft = g.field(), g.field()
    ref = []
    for x in srcs:
        g.upload_leaves(fs, x.numpy())
        g.apply_lgf(fs, ft)
        ref.append(g.download_leaves(ft))
    outs = [torch.empty((g.n_leaves, e, e, e), dtype=torch.float64).pin_memory() for _ in srcs]
    g.upload_leaves_async(fs, srcs[0])
    for k in range(len(srcs)):
        g.apply_lgf(fs, ft)
        if k + 1 < len(srcs):
            g.upload_leaves_async(fs, srcs[k + 1])
        g.download_leaves_async(ft, outs[k])
    g.synchronize()
    for r, o in zip(ref, outs):
        np.testing.assert_array_equal(o.numpy(), r)
    with pytest.raises(B.IblgfError):
        g.upload_leaves_async(fs, np.zeros((g.n_leaves, e, e, e), np.float32))


def test_async_leaf_download_checks_its_buffer():
    """The asynchronous download takes only a C-contiguous float64 host
    buffer of the leaf shape (the copy writes n_leaves e^3 doubles)."""
    case = S.GaussianPoisson("amr_small")
    g = solver(case, B.FP64)
    e = g.block_extent
    f = g.field()
    for bad in (np.zeros((g.n_leaves, e, e, e), np.float32), np.zeros((g.n_leaves, e, e, e + 1)),
                np.zeros((g.n_leaves, e, e, 2 * e))[:, :, :, ::2]):
        with pytest.raises(B.IblgfError):
            g.download_leaves_async(f, bad)
    out = np.zeros((g.n_leaves, e, e, e))
    g.download_leaves_async(f, out)
    g.synchronize()
