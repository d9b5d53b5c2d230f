"""Reader of the reference's Chombo-HDF5 field files (IO/chombo/h5_file.hpp,
chombo_impl.hpp): written from the HDF5 file-format specification, no HDF5
library needed. Covers what those files use: superblock version 0 (8-byte
offsets and lengths), version-1 object headers with continuation blocks,
version-1 group B-trees with symbol-table nodes and local heaps, attributes of
fixed-point, floating-point and string types, contiguous (and compact)
datasets of fixed-point, floating-point and compound types.

Chombo layout (chombo_impl.hpp:217-520): the root holds the attributes
num_components, num_levels, component_<i>; group level_<l> holds the
attribute dx, the compound dataset "boxes" (lo_i, lo_j, lo_k, hi_i, hi_j,
hi_k, inclusive cell ranges at that level) and "data:datatype=0", per box all
components one after the other, each over the box's cells with x fastest.
"""
import struct

import numpy as np


class H5Error(RuntimeError):
    pass


class _Obj:
    def __init__(self, addr, messages):
        self.addr = addr
        self.messages = messages  # list of (type, bytes)

    def msgs(self, t):
        return [m for (mt, m) in self.messages if mt == t]


class H5File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        b = self.b
        if b[:8] != b"\x89HDF\r\n\x1a\n":
            raise H5Error("not an HDF5 file")
        if b[8] != 0:
            raise H5Error("superblock version %d not supported" % b[8])
        self.so, self.sl = b[13], b[14]
        if self.so != 8 or self.sl != 8:
            raise H5Error("offset / length size other than 8")
        # root group symbol table entry after the 4 addresses
        root_hdr = struct.unpack_from("<Q", b, 56 + 8)[0]
        self.root = self._object(root_hdr)

    # -------------------------------------------------------------- objects
    def _object(self, addr):
        b = self.b
        ver, _, nmsg, _, hsize = struct.unpack_from("<BBHII", b, addr)
        if ver != 1:
            raise H5Error("object header version %d not supported" % ver)
        blocks = [(addr + 16, hsize)]
        messages = []
        while blocks and len(messages) < nmsg:
            start, size = blocks.pop(0)
            p, end = start, start + size
            while p + 8 <= end and len(messages) < nmsg:
                mt, ms, _flags = struct.unpack_from("<HHB", b, p)
                data = b[p + 8:p + 8 + ms]
                if mt == 0x10:  # continuation
                    off, ln = struct.unpack_from("<QQ", data, 0)
                    blocks.append((off, ln))
                messages.append((mt, data))
                p += 8 + ms
        return _Obj(addr, messages)

    def _heap_string(self, heap_addr, offset):
        b = self.b
        if b[heap_addr:heap_addr + 4] != b"HEAP":
            raise H5Error("bad local heap")
        data_addr = struct.unpack_from("<Q", b, heap_addr + 24)[0]
        s = data_addr + offset
        e = b.index(b"\0", s)
        return b[s:e].decode()

    def _btree_entries(self, addr, heap):
        b = self.b
        if b[addr:addr + 4] != b"TREE":
            raise H5Error("bad B-tree node")
        node_type, level, used = struct.unpack_from("<BBH", b, addr + 4)
        if node_type != 0:
            raise H5Error("not a group B-tree")
        out = []
        p = addr + 24 + 8  # header, first key
        for _ in range(used):
            child = struct.unpack_from("<Q", b, p)[0]
            p += 16  # child address and the next key
            if level > 0:
                out.extend(self._btree_entries(child, heap))
            else:
                if b[child:child + 4] != b"SNOD":
                    raise H5Error("bad symbol table node")
                n = struct.unpack_from("<H", b, child + 6)[0]
                q = child + 8
                for _ in range(n):
                    name_off, hdr = struct.unpack_from("<QQ", b, q)
                    out.append((self._heap_string(heap, name_off), hdr))
                    q += 40
        return out

    def members(self, obj):
        """{name: object header address} of a group."""
        st = obj.msgs(0x11)
        if not st:
            raise H5Error("not a group (no symbol table message)")
        btree, heap = struct.unpack_from("<QQ", st[0], 0)
        return dict(self._btree_entries(btree, heap))

    def get(self, obj, name):
        m = self.members(obj)
        if name not in m:
            raise H5Error("no member %r" % name)
        return self._object(m[name])

    # ------------------------------------------------------------ datatypes
    def _dtype(self, d):
        """numpy dtype of a datatype message; returns (dtype, bytes used)."""
        cv = d[0]
        cls, ver = cv & 0x0F, cv >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = struct.unpack_from("<I", d, 4)[0]
        if cls == 0:  # fixed point
            signed = bool(bits & 0x08)
            order = ">" if bits & 1 else "<"
            return np.dtype("%s%s%d" % (order, "i" if signed else "u", size)), 12
        if cls == 1:  # floating point
            order = ">" if bits & 1 else "<"
            return np.dtype("%sf%d" % (order, size)), 20
        if cls == 3:  # string
            return np.dtype("S%d" % size), 8
        if cls == 6:  # compound
            nmem = bits & 0xFFFF
            p = 8
            names, formats, offsets = [], [], []
            for _ in range(nmem):
                e = d.index(b"\0", p)
                name = d[p:e].decode()
                nl = e - p + 1
                if ver < 3:
                    p += (nl + 7) // 8 * 8
                    off = struct.unpack_from("<I", d, p)[0]
                    p += 4 + 1 + 3 + 4 + 4 + 16  # offset, dimensionality, reserved, perm, reserved, dims
                else:
                    p += nl
                    nb = 1 if size < 256 else (2 if size < 65536 else 4)
                    off = int.from_bytes(d[p:p + nb], "little")
                    p += nb
                mdt, used = self._dtype(d[p:])
                p += used
                names.append(name)
                formats.append(mdt)
                offsets.append(off)
            return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size}), p
        raise H5Error("datatype class %d not supported" % cls)

    @staticmethod
    def _dims(d):
        ver, ndim, flags = d[0], d[1], d[2]
        p = 8 if ver == 1 else 4
        dims = [struct.unpack_from("<Q", d, p + 8 * i)[0] for i in range(ndim)]
        return dims

    # ----------------------------------------------------------- attributes
    def attrs(self, obj):
        out = {}
        for d in obj.msgs(0x0C):
            ver = d[0]
            nsz, tsz, ssz = struct.unpack_from("<HHH", d, 2)
            if ver == 1:
                p = 8
                name = d[p:p + nsz].split(b"\0")[0].decode()
                p += (nsz + 7) // 8 * 8
                dt, _ = self._dtype(d[p:p + tsz])
                p += (tsz + 7) // 8 * 8
                dims = self._dims(d[p:p + ssz])
                p += (ssz + 7) // 8 * 8
            else:
                p = 8 if ver == 2 else 9
                name = d[p:p + nsz].split(b"\0")[0].decode()
                p += nsz
                dt, _ = self._dtype(d[p:p + tsz])
                p += tsz
                dims = self._dims(d[p:p + ssz])
                p += ssz
            n = int(np.prod(dims)) if dims else 1
            val = np.frombuffer(d, dtype=dt, count=n, offset=p)
            if dt.kind == "S":
                v = val[0].split(b"\0")[0].decode() if n == 1 else [x.split(b"\0")[0].decode() for x in val]
            else:
                v = val[0] if not dims else val.copy().reshape(dims)
            out[name] = v
        return out

    # -------------------------------------------------------------- datasets
    def read(self, obj):
        dt, _ = self._dtype(obj.msgs(0x03)[0])
        dims = self._dims(obj.msgs(0x01)[0])
        lay = obj.msgs(0x08)[0]
        ver = lay[0]
        n = int(np.prod(dims)) if dims else 1
        if ver == 3:
            cls = lay[1]
            if cls == 1:
                addr, size = struct.unpack_from("<QQ", lay, 2)
                if addr == 0xFFFFFFFFFFFFFFFF:
                    return np.zeros(dims, dt)
                return np.frombuffer(self.b, dtype=dt, count=n, offset=addr).copy().reshape(dims)
            if cls == 0:
                size = struct.unpack_from("<H", lay, 2)[0]
                return np.frombuffer(lay, dtype=dt, count=n, offset=4).copy().reshape(dims)
            raise H5Error("chunked datasets are not supported")
        if ver in (1, 2):
            ndim, cls = lay[1], lay[2]
            if cls != 1:
                raise H5Error("layout class %d not supported" % cls)
            addr = struct.unpack_from("<Q", lay, 8)[0]
            return np.frombuffer(self.b, dtype=dt, count=n, offset=addr).copy().reshape(dims)
        raise H5Error("layout version %d not supported" % ver)


def read_chombo(path):
    """Chombo field file -> {"components": [names], "levels": [{"dx", "boxes"
    (n, 3, 2) inclusive lo / hi per axis, "data": [per box (components, ez,
    ey, ex)]}]}."""
    f = H5File(path)
    ra = f.attrs(f.root)
    ncomp = int(np.ravel(ra["num_components"])[0])
    nlev = int(np.ravel(ra["num_levels"])[0])
    comps = [ra["component_%d" % i] for i in range(ncomp)]
    levels = []
    for l in range(nlev):
        g = f.get(f.root, "level_%d" % l)
        ga = f.attrs(g)
        boxes = f.read(f.get(g, "boxes"))
        data = f.read(f.get(g, "data:datatype=0")).astype(np.float64)
        lo = np.stack([boxes["lo_i"], boxes["lo_j"], boxes["lo_k"]], 1)
        hi = np.stack([boxes["hi_i"], boxes["hi_j"], boxes["hi_k"]], 1)
        per = []
        off = 0
        for b in range(len(lo)):
            ex, ey, ez = (hi[b] - lo[b] + 1).tolist()
            v = ex * ey * ez
            per.append(data[off:off + ncomp * v].reshape(ncomp, ez, ey, ex))
            off += ncomp * v
        if off != len(data):
            raise H5Error("box sizes do not add up to the data length")
        levels.append({"dx": float(np.ravel(ga["dx"])[0]), "boxes": np.stack([lo, hi], 2), "data": per})
    return {"components": comps, "levels": levels}


# ================================================================== writing
# The writer lays the file out bottom-up in one byte buffer: raw data and the
# object headers of a group's members first, then the group's local heap (its
# member names), symbol-table nodes, B-tree node and object header, the root
# group last; the superblock at offset 0 is filled in at the end. Structures
# follow the HDF5 file-format specification, version-0 superblock:
#   superblock 0 (offsets and lengths 8 bytes, group leaf K 4, internal K 16),
#   version-1 object headers (messages 8-byte aligned), version-1 attribute
#   messages, version-1 dataspaces (simple, max dims given; rank 0 = scalar),
#   fill value message version 2, contiguous layout message version 3,
#   group symbol tables as a one-level B-tree over symbol-table nodes of at
#   most 2K = 8 entries, names in a local heap (free list "none" = 1).

_UNDEF = 0xFFFFFFFFFFFFFFFF
_LEAF_K, _NODE_K = 4, 16


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _dt_int(size=4, signed=True):
    return struct.pack("<BBBBIHH", 0x10, 0x08 if signed else 0, 0, 0, size, 0, 8 * size)


def _dt_f64():
    # IEEE little-endian double: sign bit 63, exponent 52..62 (bias 1023),
    # mantissa 0..51 with an implied leading one
    return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)


def _dt_str(n):
    return struct.pack("<BBBBI", 0x13, 0, 0, 0, n)


def _dt_compound(members, size):
    """members: [(name, offset, member datatype bytes)], version-1 layout."""
    out = struct.pack("<BBBBI", 0x16, len(members) & 0xFF, len(members) >> 8, 0, size)
    for name, off, mdt in members:
        out += _pad8(name.encode() + b"\0")
        out += struct.pack("<IB3xI4x", off, 0, 0) + b"\0" * 16
        out += mdt
    return out


def _dataspace(dims):
    if dims is None:  # scalar
        return struct.pack("<BBBB4x", 1, 0, 0, 0)
    out = struct.pack("<BBBB4x", 1, len(dims), 1, 0)
    out += b"".join(struct.pack("<Q", d) for d in dims)
    out += b"".join(struct.pack("<Q", d) for d in dims)
    return out


def _message(mtype, body):
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), 0) + body


def _attribute(name, dt, dims, data):
    nm = name.encode() + b"\0"
    ds = _dataspace(dims)
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds))
    body += _pad8(nm) + _pad8(dt) + _pad8(ds) + data
    return _message(0x0C, body)


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)  # superblock, written last

    def _put(self, b):
        addr = len(self.buf)
        self.buf += _pad8(bytes(b))
        return addr

    def header(self, messages):
        body = b"".join(messages)
        return self._put(struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body)

    def dataset(self, dt, dims, raw, attrs=()):
        addr = self._put(raw) if len(raw) else _UNDEF
        layout = struct.pack("<BBQQ", 3, 1, addr, len(raw))
        fill = struct.pack("<BBBBI", 2, 1, 2, 1, 0)
        msgs = [_message(0x01, _dataspace(dims)), _message(0x03, dt), _message(0x05, fill), _message(0x08, layout)]
        return self.header(msgs + list(attrs))

    def group(self, members, attrs=()):
        """members: {name: (object header address, (btree, heap) or None)}.
        Returns (header address, btree address, heap address)."""
        names = sorted(members)  # symbol-table nodes hold names in byte order
        heap_data = bytearray(8)  # offset 0: the empty string
        name_off = {}
        for n in names:
            name_off[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\0")
        heap_data += b"\0" * 16  # room for one free block entry
        free_at = len(heap_data) - 16
        heap_data[free_at:free_at + 16] = struct.pack("<QQ", 1, 16)
        data_addr = self._put(bytes(heap_data))
        heap = self._put(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), free_at, data_addr))
        chunks = [names[i:i + 2 * _LEAF_K] for i in range(0, len(names), 2 * _LEAF_K)] or [[]]
        if len(chunks) > 2 * _NODE_K:
            raise H5Error("more group members than one B-tree node indexes")
        snods = []
        for ch in chunks:
            node = b"SNOD" + struct.pack("<BBH", 1, 0, len(ch))
            for n in ch:
                hdr, cache = members[n]
                if cache is None:
                    node += struct.pack("<QQI4x16x", name_off[n], hdr, 0)
                else:
                    node += struct.pack("<QQI4xQQ", name_off[n], hdr, 1, cache[0], cache[1])
            node += b"\0" * (40 * (2 * _LEAF_K - len(ch)))
            snods.append(self._put(node))
        # B-tree keys: key i bounds child i from below, key i+1 is the last
        # name of child i
        bt = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(chunks), _UNDEF, _UNDEF)
        bt += struct.pack("<Q", 0)
        for ch, sn in zip(chunks, snods):
            bt += struct.pack("<QQ", sn, name_off[ch[-1]] if ch else 0)
        bt += b"\0" * (16 * (2 * _NODE_K - len(chunks)))
        btree = self._put(bt)
        stab = _message(0x11, struct.pack("<QQ", btree, heap))
        return self.header([stab] + list(attrs)), btree, heap

    def finish(self, root):
        hdr, btree, heap = root
        sb = b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0])
        sb += struct.pack("<HHI", _LEAF_K, _NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, _UNDEF, len(self.buf), _UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, hdr, 1, btree, heap)
        self.buf[:96] = sb
        return bytes(self.buf)


def _attr_u32(name, v, n=None):
    vals = [int(v)] if n is None else [int(x) for x in v]
    return _attribute(name, _dt_int(4, signed=False), [len(vals)], struct.pack("<%dI" % len(vals), *vals))


def _attr_f64(name, v):
    return _attribute(name, _dt_f64(), [1], struct.pack("<d", float(v)))


def _attr_str(name, s):
    b = s.encode() + b"\0"
    return _attribute(name, _dt_str(len(b)), None, b)


_BOX_NAMES = ("lo_i", "lo_j", "lo_k", "hi_i", "hi_j", "hi_k")
_BOX_DT = _dt_compound([(n, 4 * i, _dt_int(4, True)) for i, n in enumerate(_BOX_NAMES)], 24)
_VEC_DT = _dt_compound([(n, 8 * i, _dt_f64()) for i, n in enumerate("xyz")], 24)


def group_blocks(keys, depth):
    """Chombo boxes of one level (chombo_impl.hpp:136-213): blocks in Morton
    order start a group when the block is child 0 of its parent and the 8
    blocks from it are consecutive Morton keys; the group grows to 64, 512
    ... blocks while the ancestor is again child 0 and the keys stay
    consecutive. `keys` are Morton indices at tree level `depth`, sorted;
    returns lists of positions into `keys`. (The reference stops growing at
    the tree level, the grouping loop's bound, and leaves no block out.)"""
    keys = [int(k) for k in keys]
    n = len(keys)
    groups = []
    i = 0
    while i < n:
        r = 0
        while r < depth:
            span = 8 ** (r + 1)
            if ((keys[i] >> (3 * r)) & 7) == 0 and i + span <= n and keys[i + span - 1] - keys[i] == span - 1 \
                    and keys[i] % span == 0:
                r += 1
            else:
                break
        size = 8 ** r
        groups.append(list(range(i, i + size)))
        i += size
    return groups


def write_chombo(path, components, levels, dx_base, time=0.0, dt=1, ref_ratio=2):
    """Writes a Chombo field file in the reference's layout
    (Chombo::write_global_metaData / write_level_info, chombo_impl.hpp:
    1755-2560): root attributes component_<i>, num_levels, num_components,
    filetype "VanillaAMRFileType", data_centering 6 and group Chombo_global
    (SpaceDim 3); per level group level_<l> the attributes dt, ghost, dx =
    dx_base / 2^l, ref_ratio, time (the reference stores dt and time as
    integers), prob_domain (bounding box of the level's boxes) and vec_dx;
    datasets "boxes" (inclusive cell ranges) and "data:datatype=0" (per box
    every component over its cells, x fastest) and group data_attributes
    (objectType "CArrayBox", dataset "offsets": 0 then each box's value count,
    as the reference fills it).

    `levels`: [{"boxes": (n, 3, 2) int, "data": [per box (components, ez,
    ey, ex)]}] as read_chombo returns them."""
    w = _Writer()
    ncomp = len(components)
    root_members = {}
    for l, lev in enumerate(levels):
        boxes = np.asarray(lev["boxes"], np.int64).reshape(-1, 3, 2)
        rec = np.zeros(len(boxes), np.dtype({"names": list(_BOX_NAMES), "formats": ["<i4"] * 6,
                                             "offsets": [0, 4, 8, 12, 16, 20], "itemsize": 24}))
        for a in range(3):
            rec[_BOX_NAMES[a]] = boxes[:, a, 0]
            rec[_BOX_NAMES[3 + a]] = boxes[:, a, 1]
        counts = [0]
        parts = []
        for b, d in zip(boxes, lev["data"]):
            d = np.asarray(d, np.float64)
            ext = tuple((b[::-1, 1] - b[::-1, 0] + 1).tolist())
            if d.shape != (ncomp,) + ext:
                raise ValueError("box data of shape %s, expected %s" % (d.shape, (ncomp,) + ext))
            parts.append(np.ascontiguousarray(d).astype("<f8").tobytes())
            counts.append(d.size)
        raw = b"".join(parts)
        members = {
            "boxes": (w.dataset(_BOX_DT, [len(boxes)], rec.tobytes()), None),
            "data:datatype=0": (w.dataset(_dt_f64(), [len(raw) // 8], raw), None),
        }
        off = w.dataset(_dt_int(4, signed=False), [len(counts)], struct.pack("<%dI" % len(counts), *counts))
        da = w.group({"offsets": (off, None)}, [_attr_str("objectType", "CArrayBox")])
        members["data_attributes"] = (da[0], da[1:])
        dx = dx_base / 2.0 ** l
        lo = boxes[:, :, 0].min(0) if len(boxes) else np.zeros(3, np.int64)
        hi = boxes[:, :, 1].max(0) if len(boxes) else np.zeros(3, np.int64)
        pd = struct.pack("<6i", *[int(v) for v in list(lo) + list(hi)])
        attrs = [_attr_u32("dt", int(dt)), _attr_u32("ghost", [1, 1, 1], 3), _attr_f64("dx", dx),
                 _attr_u32("ref_ratio", ref_ratio), _attr_u32("time", int(time)),
                 _attribute("prob_domain", _BOX_DT, [1], pd),
                 _attribute("vec_dx", _VEC_DT, [1], struct.pack("<3d", dx, dx, dx))]
        g = w.group(members, attrs)
        root_members["level_%d" % l] = (g[0], g[1:])
    cg = w.group({}, [_attr_u32("SpaceDim", 3)])
    root_members["Chombo_global"] = (cg[0], cg[1:])
    attrs = [_attr_str("component_%d" % i, c) for i, c in enumerate(components)]
    attrs += [_attr_u32("num_levels", len(levels)), _attr_u32("num_components", ncomp),
              _attr_str("filetype", "VanillaAMRFileType"), _attr_u32("data_centering", 6)]
    root = w.group(root_members, attrs)
    with open(path, "wb") as f:
        f.write(w.finish(root))


def chombo_levels(keys, levels, bbase, block_extent, base_level, values, flags=None, include_correction=False,
                  base_correction_only=True):
    """Chombo levels from octree blocks (h5_io.hpp:230-270 selection, then
    the grouping of group_blocks): every block at refinement level >= 0,
    correction blocks only with include_correction (and then only at the
    base level with base_correction_only). `values`: (n_blocks, components,
    Nb, Nb, Nb) with a one-cell buffer; the boxes hold the interior cells.
    Returns the `levels` list of write_chombo."""
    keys = np.asarray(keys, np.uint64)
    levels = np.asarray(levels)
    bbase = np.asarray(bbase).reshape(-1, 3)
    rl = levels - base_level
    keep = rl >= 0
    if flags is not None:
        corr = (np.asarray(flags) & 2) != 0
        if not include_correction:
            keep &= ~corr
        elif base_correction_only:
            keep &= ~(corr & (rl > 0))
    e = block_extent
    out = []
    for r in range(int(rl[keep].max()) + 1 if keep.any() else 0):
        sel = np.nonzero(keep & (rl == r))[0]
        depth = int(levels[sel[0]]) if len(sel) else 0
        morton = np.array([int(k) >> (64 - 3 * depth) if depth else 0 for k in keys[sel]], np.int64)
        order = np.argsort(morton, kind="stable")
        sel, morton = sel[order], morton[order]
        boxes, data = [], []
        for g in group_blocks(morton, depth):
            idx = sel[g]
            lo = bbase[idx].min(0)
            hi = bbase[idx].max(0) + e - 1
            ext = (hi - lo + 1)[::-1]
            d = np.zeros((values.shape[1],) + tuple(ext))
            for o in idx:
                s = bbase[o] - lo
                d[:, s[2]:s[2] + e, s[1]:s[1] + e, s[0]:s[0] + e] = values[o][:, 1:e + 1, 1:e + 1, 1:e + 1]
            boxes.append(np.stack([lo, hi], 1))
            data.append(d)
        out.append({"boxes": np.array(boxes).reshape(-1, 3, 2), "data": data})
    return out


def describe(path):
    """Structure of an HDF5 file as plain data: {group path: {"attrs": {name:
    [kind, shape or field names]}, "groups": [...], "datasets": {name: [kind,
    field names]}}}; kind is the numpy kind letter ("u", "i", "f", "S", "V"
    for compound)."""
    f = H5File(path)
    out = {}

    def kind(a):
        dt = np.asarray(a).dtype if not isinstance(a, str) else np.dtype("S1")
        if dt.names:
            return ["V", list(dt.names)]
        return [dt.kind, list(np.shape(a))]

    def walk(obj, p):
        ent = {"attrs": {k: kind(v) for k, v in f.attrs(obj).items()}, "groups": [], "datasets": {}}
        out[p] = ent
        for name, addr in sorted(f.members(obj).items()):
            o = f._object(addr)
            if o.msgs(0x11):
                ent["groups"].append(name)
                walk(o, p.rstrip("/") + "/" + name)
            else:
                dt, _ = f._dtype(o.msgs(0x03)[0])
                ent["datasets"][name] = ["V", list(dt.names)] if dt.names else [dt.kind, []]

    walk(f.root, "/")
    return out


def read_field_into_blocks(chombo, name, n_comp, mesh, dx_base, rl, bbase, block_extent, leaf, listed, values):
    """Chombo::read_u (chombo_impl.hpp:216-520): a field read from a Chombo
    file into octree blocks, `values` (n, n_comp, Nb, Nb, Nb) updated in
    place. The listed blocks (io::H5_io::blocks_list_build with correction
    blocks, base-level ones only) are zeroed, buffers included; then every
    listed leaf at refinement level rl[o] takes from each file box at file
    level l (runtime level fake = l + log2(dx_base / file dx of level 0),
    fake >= rl[o]) the cells over its overlap: with factor f = 2^(fake -
    rl[o]) the mean over the fine cells (f-1)/2 .. f/2 of each coarse cell
    per axis, except along the normal of a face component, the cross
    directions of an edge component and every axis of a vertex field, where
    the fine cell at offset 0 is taken. Out-of-box fine cells are skipped but
    still count in the divisor. mesh: 0 cell, 1 face, 2 edge, 3 vertex.
    `name` is the scalar's component name, or the stem of name_0, name_1,
    ... of a vector."""
    comps = chombo["components"]
    want = name + "_0" if n_comp > 1 else name
    if want not in comps:
        raise H5Error("component %r not in the file" % want)
    c0 = comps.index(want)
    values[listed] = 0.0
    if not chombo["levels"]:
        return
    diff_f = np.log2(dx_base / chombo["levels"][0]["dx"])
    if abs(round(diff_f) - diff_f) > 1e-10:
        raise H5Error("base dx doesn't match")
    diff = int(round(diff_f))
    e = block_extent
    targets = np.nonzero(listed & leaf)[0]
    for l, lev in enumerate(chombo["levels"]):
        fake = l + diff
        for box, data in zip(lev["boxes"], lev["data"]):
            flo, fhi = box[:, 0], box[:, 1]
            fext = fhi - flo + 1
            for o in targets:
                if rl[o] > fake:
                    continue
                f = 2 ** (fake - int(rl[o]))
                blo = np.asarray(bbase[o])
                # file box scaled down to the block's level (floor division
                # for either sign, BlockDescriptor::level_scale), intersected
                olo = np.maximum(blo, flo // f)
                ohi = np.minimum(blo + e - 1, fhi // f)
                if (ohi < olo).any():
                    continue
                avg = ((f - 1) // 2, f // 2)
                for k in range(n_comp):
                    win = [avg, avg, avg]
                    if mesh == 1:
                        win[k] = (0, 0)
                    elif mesh == 2:
                        win = [(0, 0)] * 3
                        win[k] = avg
                    elif mesh == 3:
                        win = [(0, 0)] * 3
                    total = float(np.prod([w[1] - w[0] + 1 for w in win]))
                    dst = values[o, k]
                    src = data[c0 + k]
                    for sz in range(win[2][0], win[2][1] + 1):
                        for sy in range(win[1][0], win[1][1] + 1):
                            for sx in range(win[0][0], win[0][1] + 1):
                                idx, pos = [], []
                                for a, s in zip(range(3), (sx, sy, sz)):
                                    ii = np.arange(olo[a], ohi[a] + 1)
                                    fi = ii * f - flo[a] + s
                                    ok = (fi >= 0) & (fi < fext[a])
                                    idx.append(fi[ok])
                                    pos.append(ii[ok] - blo[a] + 1)
                                if any(len(x) == 0 for x in idx):
                                    continue
                                dst[np.ix_(pos[2], pos[1], pos[0])] += src[np.ix_(idx[2], idx[1], idx[0])] / total
