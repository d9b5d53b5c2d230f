"""GPU parity of the immersed-boundary force solve (iblgf_ib_set_points /
iblgf_ib_solve) against the oracle's restatement of LinSysSolver::ib_solve
(linsys.hpp:113-230): IB block flags bit-identical, CG iteration count equal,
forces within 1e-9 relative L-inf in FP64 (the CG chains ~10 masked LGF and
integrating-factor solves); FP32 FFT/MAC path within 1e-4 and one iteration.
"""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("alpha", [0.0, 7e-4])
@pytest.mark.parametrize("precision,tol,dit", [(B.FP64, 1e-9, 0), (B.FP32, 1e-4, 1)])
def test_ib_solve_matches_oracle(alpha, precision, tol, dit):
    case = S.SphereIB("small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=precision)
    X = O.sphere_points(case.dx_base, o.depth - 1 - o.base_level, case.ibph)
    u = case.velocity(o)
    f_ref, flags_ref, it_ref = o.ib_solve(X, case.Re, u, alpha, 1e-3, 40)
    g.ib_set_points(X, case.Re)
    assert np.array_equal(g.ib_flags(), flags_ref)
    uf = [g.field(u[k]) for k in range(3)]
    f, it = g.ib_solve(uf, alpha, 1e-3, 40)
    assert abs(it - it_ref) <= dit, (it, it_ref)
    assert rel_linf(f, f_ref) < tol, rel_linf(f, f_ref)


def test_ib_solve_needs_points():
    case = S.SphereIB("small")
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    uf = [g.field() for _ in range(3)]
    g._ib_X = np.zeros((4, 3))
    with pytest.raises(B.IblgfError):
        g.ib_solve(uf, 0.0)


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-9), (B.FP32, 1e-4)])
def test_ns_step_with_ib_matches_oracle(precision, tol):
    """Three IF-HERK steps past the sphere in a uniform stream (frame velocity
    (-1, 0, 0): the body at rest, the fluid moving at +1): velocity, pressure
    and the three stage forces of the last step against the oracle. The first
    step runs direct, the second is captured as a CUDA graph (its force CG a
    conditional while-node) and the third replays that graph. In FP32 the
    pressure (d_i / (a33 dt), a factor 400 here) carries the FP32
    perturbation of the IB CG iterates (about 1.5e-6 of the force, so 6e-4
    for it), 1e-4 for velocity."""
    case = S.SphereIB("small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=precision)
    X = O.sphere_points(case.dx_base, o.depth - 1 - o.base_level, case.ibph)
    u0 = case.velocity(o)
    dt, fv = 0.01, (-1.0, 0.0, 0.0)
    ptol = 1e-9 if precision == B.FP64 else 1.5e-6 / (0.25 * dt)
    ur, pr, fr = o.ns_step_ib(u0, dt, case.Re, X, fv, 0.0, 3)
    g.ib_set_points(X, case.Re)
    g.ns_options(fv)
    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    T = 0.0
    for _ in range(3):
        T = g.ns_step(uf, pf, dt, case.Re, T, 1)
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < tol, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < ptol, rel_linf(g.download(pf), pr)
    for st in range(3):
        assert rel_linf(g.ib_force(st + 1), fr[st]) < tol * 10, (st, rel_linf(g.ib_force(st + 1), fr[st]))
    assert g.ib_converged() == [True, True, True]


def test_ib_solve_reports_not_converged():
    """A solve that reaches max_iter without meeting the threshold returns
    IBLGF_ENOTCONVERGED with the force and iteration count written (the
    reference's CG_solve stops there silently, linsys.hpp:202-229)."""
    case = S.SphereIB("small")
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    X = O.sphere_points(case.dx_base, g.depth - 1 - g.base_level, case.ibph)
    g.ib_set_points(X, case.Re)
    u = case.velocity(g)
    uf = [g.field(u[k]) for k in range(3)]
    with pytest.raises(B.IblgfNotConverged) as e:
        g.ib_solve(uf, 0.0, threshold=1e-15, max_iter=2)
    assert e.value.iterations == 2 and np.abs(e.value.force).max() > 0
    f, it = g.ib_solve(uf, 0.0, threshold=1e-3, max_iter=40)
    assert it < 40


def test_ns_step_with_ib_velocity_refresh_matches_oracle():
    """Velocity refresh with the immersed boundary (FP64): the correction
    stages solve the IB system from the stages' previous forces without
    replacing them (write_prev_force = false, ifherk.hpp:1476-1478), so the
    following plain step starts its CG from the same forces as the oracle."""
    case = S.SphereIB("small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=B.FP64)
    X = O.sphere_points(case.dx_base, o.depth - 1 - o.base_level, case.ibph)
    u0 = case.velocity(o)
    dt, fv, T0 = 0.01, (-1.0, 0.0, 0.0), 1.0e6
    ur, pr, fr = o.ns_step_ib(u0, dt, case.Re, X, fv, T0, 2)
    g.ib_set_points(X, case.Re)
    g.ns_options(fv)
    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    g.ns_step(uf, pf, dt, case.Re, T0, 2)
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < 1e-9, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < 1e-9, rel_linf(g.download(pf), pr)
    for st in range(3):
        assert rel_linf(g.ib_force(st + 1), fr[st]) < 1e-8, (st, rel_linf(g.ib_force(st + 1), fr[st]))
