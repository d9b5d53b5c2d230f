"""Generates tests/golden/ns_amr_lgf_ref.npz from the reference's stored
solution of its NS test (tests/ns_amr_lgf/configs/ref.hdf5 in the reference
tree: the velocity u_0..u_2 and pressure p of the single vortex ring at
T = 0.35 on dx = 0.25), read with the package's Chombo-HDF5 reader. The
fixture holds the components on the dense cell grid the file covers, indexed
by global cell index (lo = first cell per axis)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "iblgf-amr_b200"))
import chombo_h5  # noqa: E402


def source_path():
    """ref.hdf5 inside the reference tree, whose root is the first command-line
    argument or the IBLGF_REFERENCE environment variable."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IBLGF_REFERENCE")
    if not root:
        sys.exit("usage: %s <reference tree> (or set IBLGF_REFERENCE)" % sys.argv[0])
    return os.path.join(root, "tests", "ns_amr_lgf", "configs", "ref.hdf5")


def main():
    r = chombo_h5.read_chombo(source_path())
    lev = r["levels"][0]
    comps = r["components"]
    idx = [comps.index(n) for n in ("u_0", "u_1", "u_2", "p")]
    lo = lev["boxes"][:, :, 0].min(0)
    hi = lev["boxes"][:, :, 1].max(0)
    shape = tuple((hi - lo + 1)[::-1])  # (z, y, x)
    out = np.full((4,) + shape, np.nan)
    for b, data in zip(lev["boxes"], lev["data"]):
        s = b[:, 0] - lo
        e = b[:, 1] - lo + 1
        for k, c in enumerate(idx):
            out[k, s[2]:e[2], s[1]:e[1], s[0]:e[0]] = data[c]
    if np.isnan(out).any():
        raise RuntimeError("the boxes do not cover their bounding grid")
    np.savez_compressed(os.path.join(HERE, "ns_amr_lgf_ref.npz"), fields=out, lo=lo, dx=lev["dx"],
                        names=np.array(["u_0", "u_1", "u_2", "p"]))
    print("grid", shape, "lo", lo, "dx", lev["dx"], "|u|max", np.abs(out[:3]).max())


if __name__ == "__main__":
    main()
