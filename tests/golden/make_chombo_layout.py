"""Generates tests/golden/chombo_layout_ref.json: the group / attribute /
dataset structure (names and value kinds, no data) of the reference's stored
NS solution, tests/ns_amr_lgf/configs/ref.hdf5 in the reference tree, as the
package's Chombo-HDF5 reader describes it. The writer's test compares the
files it writes against this structure."""
import json
import os
import sys

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
    d = chombo_h5.describe(source_path())
    with open(os.path.join(HERE, "chombo_layout_ref.json"), "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    print(json.dumps(d, sort_keys=True)[:400])


if __name__ == "__main__":
    main()
