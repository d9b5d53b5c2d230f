"""Deterministic adaptation attempts for the adaptation tests: refine the
finest-level leaves nearest the vortex ring's centre, delete whole sibling
groups of finest-level leaves far from it (the server keeps a deletion only
when every sibling asks for it)."""
import collections

import numpy as np

import iblgf_setups as S


def ring_attempts(keys, levels, flags, bbase, base_level, block_extent, bd_base, bd_extent, refine_pct=15,
                  delete_pct=80):
    leaf, corr = (flags & 1) != 0, (flags & 2) != 0
    rl = levels - base_level
    c = (bbase + block_extent / 2) / (2.0 ** np.maximum(rl, 0))[:, None]
    cen = np.array(bd_base) + np.array(bd_extent) / 2
    r = np.linalg.norm(c - cen, axis=1)
    fin = rl.max()
    sel = leaf & ~corr & (rl == fin)
    att_k, att_l = [], []
    near = np.percentile(r[sel], refine_pct)
    for o in np.nonzero(sel & (r < near))[0]:
        att_k.append(int(keys[o]))
        att_l.append(1)
    groups = collections.defaultdict(list)
    for o in np.nonzero(sel)[0]:
        groups[S.key_parent(keys[o])].append(o)
    far = np.percentile(r[sel], delete_pct)
    for ch in groups.values():
        if len(ch) == 8 and min(r[ch]) > far:
            for o in ch:
                att_k.append(int(keys[o]))
                att_l.append(-1)
    return np.array(att_k, np.uint64), np.array(att_l, np.int32)
