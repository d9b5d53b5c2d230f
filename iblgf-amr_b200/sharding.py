"""Sharded FMM sweeps over several processes (one GPU each).

A sharded context (Solver.set_owner) computes, in every sweep, the targets its
rank owns; the sweep's level targets are then summed over the ranks by an
exchange callback before they are added into the target field, so every rank
ends the sweep with the whole result (the reference's induced-field messages
to the target's owner, decomposition/client.hpp:467-597, become one
all-reduce of the level's target blocks). Ownership follows the reference
server's load-balanced split (Server::compute_distribution,
decomposition/server.hpp:245-330), computed by the library
(Solver.partition) and restated here for host-side checks.
"""
import numpy as np


def partition(levels, flags, children, loads, n_ranks):
    """Owner rank per octant (octants in canonical order: level, then Morton
    key). levels, flags (bit 0 leaf, bit 1 correction) and children (n x 8,
    -1 for none) describe the octree, loads the per-octant load. Per level
    from the finest: the leaf and correction octants are cut in order into
    n_ranks runs of equal cumulative load (zero loads count 1); every other
    octant of the level goes to the rank of its child with the least total
    load so far (server.hpp:262-319)."""
    n = len(levels)
    load = np.asarray(loads, dtype=np.float64).copy()
    owner = np.full(n, -1, dtype=np.int64)
    total = np.zeros(n_ranks)
    for lv in range(int(levels.max()), -1, -1):
        octs = np.nonzero(levels == lv)[0]
        cand = [o for o in octs if flags[o] & 3]
        for o in cand:
            if load[o] == 0:
                load[o] = 1.0
        tl = float(sum(load[o] for o in cand))
        it, cur = 0, 0.0
        for r in range(n_ranks):
            if it >= len(octs):
                break
            target = min((r + 1) / n_ranks * tl, tl)
            count = 0
            while it < len(octs) and (cur <= target or count == 0):
                o = octs[it]
                it += 1
                if not flags[o] & 3:
                    continue
                owner[o] = r
                total[r] += load[o]
                cur += load[o]
                count += 1
        for o in octs:
            if flags[o] & 3 and owner[o] >= 0:
                continue
            best = -1
            for ch in children[o]:
                if ch < 0 or owner[ch] < 0:
                    continue
                if best < 0 or total[owner[ch]] < total[best]:
                    best = owner[ch]
            if best >= 0:
                if owner[o] >= 0:
                    total[owner[o]] -= load[o]
                owner[o] = best
                total[best] += load[o]
    owner[owner < 0] = 0
    return owner


def fmm_loads(n_infl, nbr, target_masks):
    """FmmMaskBuilder::fmm_dry's loads (fmm.hpp:597-626): per octant, its
    neighbour plus influence count for every AMR2AMR sweep in which it is a
    target (target_masks: one boolean array per sweep)."""
    nn = (np.asarray(nbr) >= 0).sum(axis=1) + np.asarray(n_infl)
    return sum(np.where(m, nn, 0) for m in target_masks).astype(np.float64)


class _DeviceArray:
    """A device buffer as a torch-importable array (CUDA array interface)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def torch_allreduce_exchange(group=None):
    """Exchange callback for Solver.set_owner: an in-place all-reduce (sum)
    of the device buffer over the process group (NCCL over NVLink for one
    GPU per process), ordered on the library's stream."""
    import torch
    import torch.distributed as dist

    def exchange(ptr, count, stream):
        t = torch.as_tensor(_DeviceArray(ptr, count), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    return exchange
