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
    ncomp = int(ra["num_components"])
    nlev = int(ra["num_levels"])
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
        levels.append({"dx": float(ga["dx"]), "boxes": np.stack([lo, hi], 2), "data": per})
    return {"components": comps, "levels": levels}
