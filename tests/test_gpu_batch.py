"""GPU parity of the batched solve (iblgf_batch_*): independent unbounded
Poisson problems of uneven size solved together must each equal the oracle's
PoissonSolver::apply_lgf (poisson.hpp:587-894) of that problem alone.
Tolerances: FP64 <= 1e-12, FP32 <= 1e-5 relative L-inf per problem."""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-12), (B.FP32, 1e-5)])
def test_batch_matches_oracle_per_problem(precision, tol):
    case = S.BatchPoisson("small")
    g = B.BatchSolver(case.block_extent, case.dx_base, case.problems, precision=precision)
    src = g.zeros()
    refs = []
    for i, p in enumerate(case.problems):
        v = g.problem(i)
        o = O.Domain(p["bd_base"], p["bd_extent"], case.block_extent, case.dx_base, p["blocks"])
        assert (o.n, o.base_level, o.depth) == (v.n, v.base_level, v.depth)
        assert np.array_equal(o.keys, v.keys) and np.array_equal(o.flags, v.flags)
        assert np.array_equal(o.bbase, v.bbase)
        src[v.offset:v.offset + v.n] = case.fields(v, i)
        refs.append(o.apply_lgf(case.fields(o, i)))
    fs, ft = g.field(src), g.field()
    for call in range(2):  # the second call reuses the merged plans and spectra
        g.apply_lgf(fs, ft)
        out = g.split(g.download(ft))
        for i, ref in enumerate(refs):
            assert rel_linf(out[i], ref) < tol, (call, i, rel_linf(out[i], ref))


def test_batch_rejects_single_problem_calls():
    case = S.BatchPoisson("small")
    g = B.BatchSolver(case.block_extent, case.dx_base, case.problems[:2])
    f = g.field()
    with pytest.raises(B.IblgfError):
        g.fmm_apply(f, f, g.problem(0).base_level, 1)
    with pytest.raises(B.IblgfError):
        B.Solver.apply_lgf(g, f, f)
    L = B.lib()
    assert L.iblgf_domain_add_blocks(g.h, 0, None, None) != 0
