"""GPU parity of the IF-HERK time step (ifherk.hpp:1078-1200) against the
oracle's restatement, through the C ABI (iblgf_ns_step).

Two steps of the small vortex-ring flow; every node of every block of the
three velocity components and of the pressure is compared. Tolerances:
FP64 <= 1e-10 relative L-inf (the step chains ~20 Poisson / integrating-factor
solves), FP32 FFT/MAC path <= 1e-5.
"""
import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-10), (B.FP32, 1e-5)])
def test_ns_step_matches_oracle(precision, tol):
    case = S.VortexRingNS("small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=precision)
    assert np.array_equal(o.keys, g.keys) and np.array_equal(o.flags, g.flags)
    u0 = case.initial_velocity(o)
    dt = case.dt()
    ur, pr = o.ns_step(u0, dt, case.Re, 0.0, 2)
    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    T = g.ns_step(uf, pf, dt, case.Re, 0.0, 2)
    assert abs(T - 2 * dt) < 1e-14
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < tol, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < tol, rel_linf(g.download(pf), pr)


def test_ns_step_rejects_bad_arguments():
    case = S.VortexRingNS("small")
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    uf = [g.field() for _ in range(3)]
    pf = g.field()
    with pytest.raises(B.IblgfError):
        g.ns_step(uf, pf, -1.0, case.Re, 0.0, 1)
    with pytest.raises(B.IblgfError):
        g.ns_step([uf[0], uf[1], 999], pf, case.dt(), case.Re, 0.0, 1)
    with pytest.raises(B.IblgfError):
        g.ns_step(uf, pf, case.dt(), 0.0, 0.0, 1)


@pytest.mark.parametrize("precision,tol", [(B.FP64, 1e-10), (B.FP32, 1e-5)])
def test_ns_step_velocity_refresh_matches_oracle(precision, tol):
    """Velocity refresh (ifherk.hpp:1093-1111): with T far past the last
    refresh, the first step rebuilds u through the stream function on the base
    level (pad_velocity) and runs the alpha = 0 correction step before its
    stages; the second step is a plain one. Velocity and pressure against the
    oracle, same tolerances as the plain steps."""
    case = S.VortexRingNS("small")
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=precision)
    u0 = case.initial_velocity(o)
    dt, T0 = case.dt(), 1.0e6
    assert (T0 / (case.Re * case.dx_base ** 2)) * 3.3 > 7 > (dt / (case.Re * case.dx_base ** 2)) * 3.3
    ur, pr = o.ns_step(u0, dt, case.Re, T0, 2)
    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    T = g.ns_step(uf, pf, dt, case.Re, T0, 2)
    assert abs(T - (T0 + 2 * dt)) < 1e-6
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < tol, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < tol, rel_linf(g.download(pf), pr)
