"""Sharded sweeps on the device (one GPU, two ranks emulated by two
contexts driven from two host threads; they share no device work and meet
only in the host-side exchange).

* The library's partition equals the host restatement (sharding.partition).
* Each context computes only its rank's targets; the exchange callback sums
  the two ranks' level-target buffers (downloaded, added on the host,
  uploaded) like an all-reduce; the sharded apply_lgf (every level, both
  sweeps, correction) and an IF-HERK-free Fmm sweep per level equal the
  unsharded context's results: FP64 <= 1e-12 relative L-inf.
"""
import threading

import numpy as np
import pytest

import iblgf_b200 as B
import iblgf_setups as S
import sharding

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _solver(case):
    return B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                    n_levels=case.n_levels, predicate=case.predicate)


class _HostAllReduce:
    """All-reduce of two ranks' device buffers through host memory."""

    def __init__(self, world):
        import torch
        self.torch = torch
        self.world = world
        self.barrier = threading.Barrier(world)
        self.parts = [None] * world
        self.calls = 0

    def callback(self, rank):
        torch = self.torch

        def exchange(ptr, count, stream):
            t = torch.as_tensor(sharding._DeviceArray(ptr, count), device="cuda")
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                self.parts[rank] = t.cpu().numpy().copy()  # waits for the stream
                self.barrier.wait(timeout=120)
                total = self.parts[0] + self.parts[1]  # rank order fixed: identical on both ranks
                self.barrier.wait(timeout=120)
                t.copy_(torch.from_numpy(total))
                torch.cuda.current_stream().synchronize()
            if rank == 0:
                self.calls += 1

        return exchange


def test_partition_matches_host_restatement():
    case = S.GaussianPoisson("amr_small")
    g = _solver(case)
    nbr, infl, ni = g.lists()
    masks = [g.masks(15 + 2 * rl + nlas)[:, 1] != 0 for rl in range(g.depth - g.base_level) for nlas in (0, 1)]
    loads = sharding.fmm_loads(ni, nbr, masks)
    key_index = {int(k): i for i, k in enumerate(g.keys)}
    children = np.full((g.n, 8), -1)
    fill = np.zeros(g.n, dtype=int)
    for i, k in enumerate(g.keys):
        if g.levels[i] == 0:
            continue
        k = int(k)
        lv = (k & 0x7C) >> 2
        mask = 0 if lv - 1 <= 0 else (((1 << (3 * (lv - 1))) - 1) << (64 - 3 * (lv - 1)))
        p = key_index.get(((mask & k) | ((lv - 1) << 2)) + 1, -1)
        if p >= 0:
            children[p, fill[p]] = i
            fill[p] += 1
    for n in (2, 3):
        assert np.array_equal(g.partition(n), sharding.partition(g.levels, g.flags, children, loads, n))


@pytest.mark.parametrize("what", ["apply_lgf", "fmm_apply"])
def test_two_rank_sharded_solve_matches_single(what):
    case = S.GaussianPoisson("amr_small")
    full = _solver(case)
    src = case.fields(full)
    fs, ft = full.field(src), full.field()
    ranks = [_solver(case) for _ in range(2)]
    owner = full.partition(2)
    assert set(np.unique(owner)) == {0, 1}
    ex = _HostAllReduce(2)
    for r, g in enumerate(ranks):
        g.set_owner(owner, r, ex.callback(r))
    fields = [(g.field(src), g.field()) for g in ranks]
    levels = range(full.base_level, full.depth)

    def run(g, s, t):
        if what == "apply_lgf":
            g.apply_lgf(s, t)
        else:
            for lv in levels:
                g.fmm_apply(s, t, lv, 1, 0.5)

    run(full, fs, ft)
    ref = full.download(ft)
    errors = []

    def rank_main(r):
        try:
            run(ranks[r], *fields[r])
        except Exception as e:  # surfaced below
            errors.append(e)
            ex.barrier.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errors, errors
    assert ex.calls > 0
    for r, g in enumerate(ranks):
        out = g.download(fields[r][1])
        assert rel_linf(out, ref) < 1e-12, (r, rel_linf(out, ref))
