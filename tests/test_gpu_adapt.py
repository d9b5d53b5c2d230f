"""GPU parity of the mesh adaptation (iblgf_adapt: Ifherk::adapt,
ifherk.hpp:1018-1076, with the server side of Domain::adapt,
decomposition.hpp:182-470) against the oracle's restatement, on the small
vortex-ring domain with deterministic attempts (refine near the ring, delete
whole far sibling groups):

* the adapted octree (keys, levels, leaf / correction flags) is identical;
* every field keeps its values on the octants that stay (bit-exact) and the
  listed face velocity is interpolated into new children (<= 1e-13);
* a Poisson solve and an IF-HERK step (velocity refresh, as after a base mesh
  update) on the adapted tree agree with the oracle (FP64, <= 1e-12 / 1e-10);
* the block norms behind the adapt condition equal a numpy evaluation.
"""
import numpy as np
import pytest

import adapt_cases as A
import iblgf_b200 as B
import iblgf_setups as S
import oracle_lib as O

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make(case):
    o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=B.FP64)
    return o, g


def test_adapt_matches_oracle():
    case = S.VortexRingNS("small")
    o, g = make(case)
    att_k, att_l = A.ring_attempts(o.keys, o.levels, o.flags, o.bbase, o.base_level, o.block_extent,
                                   case.bd_base, case.bd_extent)
    u0 = case.initial_velocity(o)
    rnd = np.random.default_rng(5).standard_normal((o.n, o.Nb, o.Nb, o.Nb))
    uf = [g.field(u0[k]) for k in range(3)]
    rf = g.field(rnd)
    bmu_g = g.adapt(att_k, att_l, interpolate=[(1, uf)])
    bmu_o, (ux, uy, uz, rn) = o.adapt(att_k, att_l, [(u0[0], 1, 0), (u0[1], 1, 1), (u0[2], 1, 2), (rnd, -1, 0)])
    assert bmu_g == bmu_o
    assert g.n == o.n and g.depth == o.depth
    assert np.array_equal(g.keys, o.keys) and np.array_equal(g.levels, o.levels)
    assert np.array_equal(g.flags, o.flags)
    assert np.array_equal(g.download(rf), rn)
    for k, ref in enumerate((ux, uy, uz)):
        assert rel_linf(g.download(uf[k]), ref) < 1e-13, (k, rel_linf(g.download(uf[k]), ref))
    # a Poisson solve on the adapted tree
    src = np.random.default_rng(6).standard_normal((o.n, o.Nb, o.Nb, o.Nb))
    src[:, [0, -1], :, :] = 0
    src[:, :, [0, -1], :] = 0
    src[:, :, :, [0, -1]] = 0
    tgt_o = o.apply_lgf(src)
    fs, ft = g.field(src), g.field()
    g.apply_lgf(fs, ft)
    assert rel_linf(g.download(ft), tgt_o) < 1e-12, rel_linf(g.download(ft), tgt_o)
    # an IF-HERK step with the velocity refresh on the adapted tree
    dt, T0 = case.dt(), 1.0e6
    ur, pr = o.ns_step(np.stack([ux, uy, uz]), dt, case.Re, T0, 1)
    pf = g.field()
    g.ns_step(uf, pf, dt, case.Re, T0, 1)
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < 1e-10, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < 1e-10


def test_block_norms_match_numpy():
    case = S.VortexRingNS("small")
    o, g = make(case)
    u0 = case.initial_velocity(o)
    uf = [g.field(u0[k]) for k in range(3)]
    mx, rms = g.block_norms(uf)
    inner = u0[:, :, 1:-1, 1:-1, 1:-1]
    mag2 = (inner ** 2).sum(0).reshape(o.n, -1)
    assert np.allclose(mx, np.sqrt(mag2.max(1)), rtol=1e-14, atol=0)
    assert np.allclose(rms, np.sqrt(mag2.mean(1)), rtol=1e-13, atol=0)
    with pytest.raises(B.IblgfError):
        g.block_norms([uf[0], uf[1], uf[2], uf[0]])


def test_ns_march_with_adaptation_matches_oracle_replay():
    """Ifherk::time_march with adaptation (adapt_frequency 2): three
    iterations, the third preceded by an adaptation whose attempts come from
    the NS setup's adapt condition (ns_amr_lgf.hpp:402-489) on the device's
    block norms; the oracle replays the same sequence (two steps, the same
    attempts with the velocity interpolated, one step, a grown base mesh
    refreshing the velocity and the former correction blocks cleaned as such
    for that step). Velocity and pressure, FP64, <= 1e-10."""
    case = S.VortexRingNS("small")
    o, g = make(case)
    u0 = case.initial_velocity(o)
    dt = case.dt()

    def cond(sv, mc, mk, me, sm):
        return S.adapt_level_change(sv.keys, sv.levels, sv.flags, sv.base_level, mc, mk, me, sm,
                                    n_level_refinement=sv.depth - sv.base_level)

    uf = [g.field(u0[k]) for k in range(3)]
    pf = g.field()
    n0 = g.n
    T, sm, hist = g.ns_march(uf, pf, dt, case.Re, 0.0, 3, adapt_freq=2, adapt_condition=cond)
    assert len(hist) == 1 and len(hist[0][0]) > 0 and g.n != n0
    assert abs(T - 3 * dt) < 1e-14
    uo, _ = o.ns_step(u0, dt, case.Re, 0.0, 2)
    _, (ux, uy, uz) = o.adapt(hist[0][0], hist[0][1], [(uo[0], 1, 0), (uo[1], 1, 1), (uo[2], 1, 2)])
    assert np.array_equal(g.keys, o.keys) and np.array_equal(g.flags, o.flags)
    ur, pr = o.ns_step(np.stack([ux, uy, uz]), dt, case.Re, 2 * dt, 1)
    for k in range(3):
        assert rel_linf(g.download(uf[k]), ur[k]) < 1e-10, (k, rel_linf(g.download(uf[k]), ur[k]))
    assert rel_linf(g.download(pf), pr) < 1e-10, rel_linf(g.download(pf), pr)
