"""Restart files through the C ABI (Ifherk::write_restart, ifherk.hpp:428-444;
Domain restart, domain.hpp:235-290 with restart_list_construct :839-849;
Chombo::read_u, chombo_impl.hpp:216-520): the vortex ring of the reference's
NS test (configFile_1, two levels) after 2 IF-HERK steps is written as
restart_field.hdf5 + tree_info.bin + restart_info, a new solver rebuilds the
octree from tree_info.bin alone (the correction flags recomputed) and reads
the velocity and pressure back into its leaves."""
import os

import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S

pytestmark = pytest.mark.gpu


def vortex_ring(case, g):
    w = case.initial_vorticity(g)
    wf = [g.field(w[k]) for k in range(3)]
    sf = [g.field() for _ in range(3)]
    for k in range(3):
        g.apply_lgf(wf[k], sf[k])
    uf = [g.field() for _ in range(3)]
    for lv in range(g.base_level, g.depth):
        g.op(4, sf, uf, lv, -1.0)
        for k in range(3):
            g.buffer_exchange(uf[k], lv)
    return uf


def test_restart_round_trip(tmp_path):
    case = S.NsAmrLgfTest(1)
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=B.FP64)
    uf = vortex_ring(case, g)
    pf = g.field()
    T, sm, _ = g.ns_march(uf, pf, case.dt, case.Re, 0.0, 2)
    d = str(tmp_path)
    g.write_restart(d, [("u", uf), ("p", pf)], T, adapt_count=0, source_max=sm)
    info = B.read_restart_info(os.path.join(d, "restart_info"))
    assert info["T"] == T and info["cell_aux_max"] == sm[0]

    r = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, None,
                 precision=B.FP64, restart_tree=os.path.join(d, "tree_info.bin"))
    assert (r.base_level, r.depth, r.n) == (g.base_level, g.depth, g.n)
    np.testing.assert_array_equal(r.keys, g.keys)
    np.testing.assert_array_equal(r.levels, g.levels)
    np.testing.assert_array_equal(r.flags, g.flags)  # leaf and the recomputed correction flags
    np.testing.assert_array_equal(r.bbase, g.bbase)
    ru = [r.field() for _ in range(3)]
    rp = r.field()
    path = os.path.join(d, "restart_field.hdf5")
    r.read_chombo_field(path, "u", ru, mesh=1)
    r.read_chombo_field(path, "p", rp, mesh=0)
    leaf = g.leaf
    for a, b in list(zip(uf, ru)) + [(pf, rp)]:
        x = g.download(a)[:, 1:-1, 1:-1, 1:-1]
        y = r.download(b)[:, 1:-1, 1:-1, 1:-1]
        np.testing.assert_array_equal(x[leaf], y[leaf])
        assert not y[~leaf].any()
