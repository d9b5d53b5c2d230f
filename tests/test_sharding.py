"""Sharded sweeps, host side, on CPU with two gloo ranks (no GPU).

Each rank computes the reference server's load-balanced partition
(sharding.partition, Server::compute_distribution restated) from the
oracle's octree, lists and masks; the two ranks must agree on it, every
octant has one owner, each level's leaf / correction octants form one
contiguous run per rank in Morton order, and the loads balance to within one
octant's load. The exchange: for every level, each rank keeps the oracle's
sweep result on the level targets it owns (zeros elsewhere), and the
all-reduce over the ranks gives back the whole sweep result exactly.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "iblgf-amr_b200"))
    import torch.distributed as dist

    import iblgf_setups as S
    import oracle_lib as O
    import sharding
    try:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
        case = S.GaussianPoisson("amr_small")
        o = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                     n_levels=case.n_levels, predicate=case.predicate)
        nbr, infl, ni = o.lists()
        masks = [o.masks(15 + 2 * rl + nlas)[:, 1] != 0 for rl in range(o.depth - o.base_level)
                 for nlas in (0, 1)]
        loads = sharding.fmm_loads(ni, nbr, masks)
        key_index = {int(k): i for i, k in enumerate(o.keys)}
        children = np.full((o.n, 8), -1)
        fill = np.zeros(o.n, dtype=int)
        for i, k in enumerate(o.keys):
            if o.levels[i] == 0:
                continue
            p = key_index.get(_parent_key(int(k)), -1)
            if p >= 0:
                children[p, fill[p]] = i
                fill[p] += 1
        owner = sharding.partition(o.levels, o.flags, children, loads, world)
        allo = [torch.zeros(o.n, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(allo, torch.from_numpy(owner))
        assert all(torch.equal(a, allo[0]) for a in allo)
        assert owner.min() >= 0 and owner.max() < world
        rng = np.random.default_rng(1)
        src = rng.standard_normal((o.n, o.Nb, o.Nb, o.Nb))
        worst = 0.0
        for level in range(o.base_level, o.depth):
            full = o.fmm_apply(src, o.zeros(), level, 1, 1.0, 1)
            mine = np.where(((o.levels == level) & (owner == rank))[:, None, None, None], full, 0.0)
            t = torch.from_numpy(mine.copy())
            dist.all_reduce(t)
            lvl = o.levels == level
            worst = max(worst, float(np.abs(t.numpy()[lvl] - full[lvl]).max()))
        q.put((rank, "ok", owner.tolist(), worst, o.levels.tolist(), o.flags.tolist(), loads.tolist()))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e), 0, 0, 0, 0))


def _parent_key(key):
    # keys.hpp key_parent: keep the coordinate bits of levels < l, level l - 1
    lv = (key & 0x7C) >> 2
    mask = 0 if lv - 1 <= 0 else (((1 << (3 * (lv - 1))) - 1) << (64 - 3 * (lv - 1)))
    return ((mask & key) | ((lv - 1) << 2)) + 1


def test_two_rank_partition_and_exchange():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    res.sort()
    for r in res:
        assert r[1] == "ok", r
    owner, worst = np.array(res[0][2]), max(r[3] for r in res)
    levels, flags, loads = np.array(res[0][4]), np.array(res[0][5]), np.array(res[0][6])
    assert worst == 0.0  # each block has exactly one nonzero contribution
    for lv in np.unique(levels):
        cand = np.nonzero((levels == lv) & ((flags & 3) != 0))[0]
        seq = owner[cand]
        assert np.all(np.diff(seq) >= 0), lv  # contiguous runs in Morton order
    cand = (flags & 3) != 0
    per = [loads[cand & (owner == r)].sum() for r in range(2)]
    assert abs(per[0] - per[1]) <= 2 * loads[cand].max() + 1e-9
