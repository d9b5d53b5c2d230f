"""Chombo-HDF5 writer (IO/chombo/chombo_impl.hpp, h5_file.hpp): files written
by chombo_h5.write_chombo read back through the package's reader, carry the
structure of the reference's own stored file, and group blocks into boxes as
the reference's Chombo::init does."""
import json
import os

import numpy as np
import pytest

import chombo_h5 as C

HERE = os.path.dirname(os.path.abspath(__file__))


def key_make(x, y, z, level):
    """Morton key of the reference octree (octree/key.hpp): coordinates
    interleaved from bit 63 down, level at bits [2, 7), bit 0 set."""
    idx = 0
    for b in range(21):
        idx |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2)
    return ((idx << 7) << (3 * (19 - level))) & (2 ** 64 - 1) | (level << 2) | 1


def _random_levels(rng, n_levels, ncomp):
    levels = []
    for l in range(n_levels):
        boxes, data = [], []
        for _ in range(int(rng.integers(1, 5))):
            lo = rng.integers(-20, 20, 3)
            ext = rng.integers(1, 7, 3)
            boxes.append(np.stack([lo, lo + ext - 1], 1))
            data.append(rng.standard_normal((ncomp,) + tuple(ext[::-1])))
        levels.append({"boxes": np.array(boxes), "data": data})
    return levels


@pytest.mark.parametrize("n_levels", [1, 3, 11])
def test_write_read_round_trip(tmp_path, n_levels):
    rng = np.random.default_rng(7 + n_levels)
    comps = ["cell_aux", "u_0", "u_1", "u_2", "p"]
    levels = _random_levels(rng, n_levels, len(comps))
    path = str(tmp_path / "f.hdf5")
    C.write_chombo(path, comps, levels, dx_base=0.25, time=3.7, dt=1)
    r = C.read_chombo(path)
    assert r["components"] == comps
    assert len(r["levels"]) == n_levels
    for l, (a, b) in enumerate(zip(levels, r["levels"])):
        assert b["dx"] == 0.25 / 2 ** l
        np.testing.assert_array_equal(a["boxes"], b["boxes"])
        for x, y in zip(a["data"], b["data"]):
            np.testing.assert_array_equal(x, y)


def test_structure_matches_reference_file(tmp_path):
    """Same groups, datasets and attributes (names and value kinds) as the
    reference's stored NS solution; the reference's current writer adds the
    level attributes ghost and vec_dx, which that older file lacks."""
    ref = json.load(open(os.path.join(HERE, "golden", "chombo_layout_ref.json")))
    rng = np.random.default_rng(1)
    comps = ["cell_aux", "edge_aux_0", "edge_aux_1", "edge_aux_2", "u_0", "u_1", "u_2", "p"]
    path = str(tmp_path / "f.hdf5")
    C.write_chombo(path, comps, _random_levels(rng, 1, len(comps)), dx_base=0.25)
    got = C.describe(path)
    assert sorted(got) == sorted(ref)
    for p in ref:
        assert got[p]["groups"] == ref[p]["groups"], p
        assert got[p]["datasets"] == ref[p]["datasets"], p
        extra = set(got[p]["attrs"]) - set(ref[p]["attrs"])
        assert extra <= {"ghost", "vec_dx"}, (p, extra)
        for k, v in ref[p]["attrs"].items():
            assert got[p]["attrs"][k] == v, (p, k)
    f = C.H5File(path)
    la = f.attrs(f.get(f.root, "level_0"))
    assert list(la["ghost"]) == [1, 1, 1] and tuple(la["vec_dx"][0]) == (0.25, 0.25, 0.25)
    ra = f.attrs(f.root)
    assert ra["filetype"] == "VanillaAMRFileType" and list(ra["data_centering"]) == [6]


def test_group_blocks():
    assert C.group_blocks(range(8), 2) == [list(range(8))]
    assert C.group_blocks(range(64), 3) == [list(range(64))]
    # the ancestor at each step must be child 0: 8..71 is not a 64-group
    g = C.group_blocks(range(8, 72), 3)
    assert [len(x) for x in g] == [8] * 8
    # 0..6 have no complete sibling set; 8..15 do
    g = C.group_blocks(list(range(7)) + list(range(8, 16)), 2)
    assert [len(x) for x in g] == [1] * 7 + [8]
    # a level with every block of the tree level groups up to that level
    assert C.group_blocks(range(64), 2) == [list(range(64))]


def test_chombo_levels_places_cells():
    """Blocks of a two-level octree (a 4^3 base of extent 4, one base block
    refined) with values = a function of the global cell index: every box
    holds that function over its cells, the boxes tile the blocks, correction
    blocks are left out."""
    e, nb = 4, 6
    base = 2
    keys, levels, bbase, flags = [], [], [], []
    for z in range(4):
        for y in range(4):
            for x in range(4):
                keys.append(key_make(x, y, z, base))
                levels.append(base)
                bbase.append((x * e, y * e, z * e))
                flags.append(1 if (x, y, z) != (1, 1, 1) else 0)
    for c in range(8):
        x, y, z = 2 + (c & 1), 2 + (c >> 1 & 1), 2 + (c >> 2)
        keys.append(key_make(x, y, z, base + 1))
        levels.append(base + 1)
        bbase.append((x * e, y * e, z * e))
        flags.append(1)
    flags[0] |= 2  # one correction block at the base level
    keys, levels, bbase, flags = map(np.array, (keys, levels, bbase, flags))

    def fn(l, x, y, z):
        return 1e6 * l + x + 100 * y + 10000 * z

    vals = np.zeros((len(keys), 2, nb, nb, nb))
    for o in range(len(keys)):
        zz, yy, xx = np.meshgrid(*[np.arange(-1, e + 1) + bbase[o][a] for a in (2, 1, 0)], indexing="ij")
        vals[o, 0] = fn(levels[o] - base, xx, yy, zz)
        vals[o, 1] = -vals[o, 0]
    out = C.chombo_levels(keys, levels, bbase, e, base, vals, flags)
    assert len(out) == 2
    n_cells = [0, 0]
    for l, lev in enumerate(out):
        for b, d in zip(lev["boxes"], lev["data"]):
            zz, yy, xx = np.meshgrid(*[np.arange(b[a, 0], b[a, 1] + 1) for a in (2, 1, 0)], indexing="ij")
            np.testing.assert_array_equal(d[0], fn(l, xx, yy, zz))
            np.testing.assert_array_equal(d[1], -d[0])
            n_cells[l] += xx.size
    assert n_cells == [63 * e ** 3, 8 * e ** 3]
    assert len(out[1]["boxes"]) == 1  # the 8 children form one box
    # with the correction block included it is one more block at the base
    out = C.chombo_levels(keys, levels, bbase, e, base, vals, flags, include_correction=True)
    assert sum(np.prod(b[:, 1] - b[:, 0] + 1) for b in out[0]["boxes"]) == 64 * e ** 3


def _two_level_tree():
    """A 4^3 base of blocks of extent 4 at tree level 2 with base block
    (1, 1, 1) refined (8 children at level 3); block (0, 0, 0) a base-level
    correction block."""
    e, base = 4, 2
    keys, levels, bbase, flags = [], [], [], []
    for z in range(4):
        for y in range(4):
            for x in range(4):
                keys.append(key_make(x, y, z, base))
                levels.append(base)
                bbase.append((x * e, y * e, z * e))
                flags.append(1 if (x, y, z) != (1, 1, 1) else 0)
    for c in range(8):
        x, y, z = 2 + (c & 1), 2 + (c >> 1 & 1), 2 + (c >> 2)
        keys.append(key_make(x, y, z, base + 1))
        levels.append(base + 1)
        bbase.append((x * e, y * e, z * e))
        flags.append(1)
    flags[0] |= 2
    return e, base, np.array(keys, np.uint64), np.array(levels), np.array(bbase), np.array(flags)


@pytest.mark.parametrize("mesh", [0, 1, 2, 3])
def test_read_field_round_trip(tmp_path, mesh):
    """A field written with write_chombo and read back with the read_u
    restatement returns every leaf's interior unchanged (factor 1); the
    buffers of listed blocks and the non-leaf blocks come back zero."""
    e, base, keys, levels, bbase, flags = _two_level_tree()
    nb = e + 2
    rng = np.random.default_rng(mesh)
    n_comp = 1 if mesh in (0, 3) else 3
    vals = rng.standard_normal((len(keys), n_comp, nb, nb, nb))
    levs = C.chombo_levels(keys, levels, bbase, e, base, vals, flags, include_correction=True)
    names = ["w"] if n_comp == 1 else ["w_0", "w_1", "w_2"]
    path = str(tmp_path / "f.hdf5")
    C.write_chombo(path, ["other"] + names, [{"boxes": l["boxes"], "data": [np.concatenate(
        [np.zeros((1,) + d.shape[1:]), d]) for d in l["data"]]} for l in levs], dx_base=0.5)
    rl = levels - base
    leaf = (flags & 1) != 0
    listed = (rl >= 0) & (((flags & 2) == 0) | (rl == 0))
    got = np.full_like(vals, 7.0)
    C.read_field_into_blocks(C.read_chombo(path), "w", n_comp, mesh, 0.5, rl, bbase, e, leaf, listed, got)
    inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    for o in range(len(keys)):
        if leaf[o]:
            np.testing.assert_array_equal(got[o][inner], vals[o][inner])
            g = got[o].copy()
            g[inner] = 0
            assert not g.any()
        else:
            assert not got[o].any()


@pytest.mark.parametrize("mesh", [0, 1, 2])
def test_read_field_from_finer_file(tmp_path, mesh):
    """A file whose level 0 is one level finer than the runtime base
    (dx_base / 2): each base leaf cell takes the mean of its 2x2x2 fine
    cells (cell), of the 2x2 fine faces at offset 0 along the normal (face)
    or of the 2 fine edges along the edge at offset 0 across it (edge)."""
    rng = np.random.default_rng(10 + mesh)
    n_comp = 1 if mesh == 0 else 3
    fine = rng.standard_normal((n_comp, 16, 16, 16))  # (c, z, y, x) over cells 0..15
    path = str(tmp_path / "f.hdf5")
    C.write_chombo(path, ["q"] if n_comp == 1 else ["q_0", "q_1", "q_2"],
                   [{"boxes": np.array([[[0, 15], [0, 15], [0, 15]]]), "data": [fine]}], dx_base=0.25)
    e, nb = 4, 6
    keys = [key_make(x, y, z, 1) for z in range(2) for y in range(2) for x in range(2)]
    bbase = np.array([(x * e, y * e, z * e) for z in range(2) for y in range(2) for x in range(2)])
    rl = np.zeros(8, int)
    leaf = np.ones(8, bool)
    got = np.zeros((8, n_comp, nb, nb, nb))
    C.read_field_into_blocks(C.read_chombo(path), "q", n_comp, mesh, 0.5, rl, bbase, e, leaf, leaf, got)
    for o in range(8):
        for k in range(n_comp):
            win = [(0, 1)] * 3
            if mesh == 1:
                win[k] = (0, 0)
            elif mesh == 2:
                win = [(0, 0)] * 3
                win[k] = (0, 1)
            exp = np.zeros((e, e, e))
            cnt = 0
            for sz in range(win[2][0], win[2][1] + 1):
                for sy in range(win[1][0], win[1][1] + 1):
                    for sx in range(win[0][0], win[0][1] + 1):
                        b = bbase[o]
                        exp += fine[k, 2 * b[2] + sz:2 * b[2] + 2 * e:2, 2 * b[1] + sy:2 * b[1] + 2 * e:2,
                                    2 * b[0] + sx:2 * b[0] + 2 * e:2]
                        cnt += 1
            np.testing.assert_allclose(got[o, k, 1:-1, 1:-1, 1:-1], exp / cnt, rtol=0, atol=1e-15)


def test_tree_file_round_trip(tmp_path):
    import iblgf_b200 as B
    e, base, keys, levels, bbase, flags = _two_level_tree()
    # ancestors with data, as the octree holds them, and the root
    extra = [key_make(0, 0, 0, 0), key_make(0, 0, 0, 1), key_make(1, 1, 1, 1)]
    k = np.concatenate([keys, np.array(extra, np.uint64)])
    lv = np.concatenate([levels, [0, 1, 1]])
    fl = np.concatenate([flags, [0, 0, 0]])
    path = str(tmp_path / "tree_info.bin")
    B.write_tree(path, k, lv, fl)
    assert os.path.getsize(path) == 9 * (len(k) - 1)
    rk, rleaf = B.read_tree(path)
    assert list(rk) == sorted(int(x) for x in k if (int(x) >> 2) & 31 > 0)
    m = {int(a): int(f) & 1 for a, f in zip(k, fl)}
    assert [m[int(a)] for a in rk] == list(rleaf)
    # depth-first: every octant precedes its descendants, siblings in child order
    assert list(rk).index(key_make(0, 0, 0, 1)) < list(rk).index(key_make(0, 0, 0, 2))


def test_restart_info_round_trip(tmp_path):
    import iblgf_b200 as B
    p = tmp_path / "restart_info"
    p.write_text("T = 0.35000000000000003;\nadapt_count = 3;\ncell_aux_max = 1.5;\nu_max = 2;\n"
                 "restart_n_last = 7;\nT_last_vel_refresh = 0.25;\n")
    d = B.read_restart_info(str(p))
    assert d == {"T": 0.35000000000000003, "adapt_count": 3, "cell_aux_max": 1.5, "u_max": 2,
                 "restart_n_last": 7, "T_last_vel_refresh": 0.25}


def test_read_field_factor_four_window(tmp_path):
    """A file two levels finer than the runtime base (dx_base / 4): read_u's
    window per axis is fine offsets (4-1)/2 .. 4/2 = 1..2 of each coarse
    cell, so a cell field reads the mean of the central 2x2x2 of its 4x4x4
    fine cells."""
    rng = np.random.default_rng(21)
    fine = rng.standard_normal((1, 16, 16, 16))
    path = str(tmp_path / "f.hdf5")
    C.write_chombo(path, ["q"], [{"boxes": np.array([[[0, 15], [0, 15], [0, 15]]]), "data": [fine]}],
                   dx_base=0.25)
    e = 4
    got = np.zeros((1, 1, e + 2, e + 2, e + 2))
    one = np.ones(1, bool)
    C.read_field_into_blocks(C.read_chombo(path), "q", 1, 0, 1.0, np.zeros(1, int), np.zeros((1, 3), int), e, one,
                             one, got)
    exp = np.zeros((e, e, e))
    for sz in (1, 2):
        for sy in (1, 2):
            for sx in (1, 2):
                exp += fine[0, sz::4, sy::4, sx::4]
    np.testing.assert_allclose(got[0, 0, 1:-1, 1:-1, 1:-1], exp / 8, rtol=0, atol=1e-15)
