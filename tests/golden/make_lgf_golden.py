"""Generate tests/golden/lgf_table_sample.json from the reference's own LGF
table generator (include/iblgf/lgf/lgf_table_gen/lgf_integrator.py, scipy
quad), which is what produced the reference's missing lgf_gl_lookup.cpp table
(python_lgf.py:9-21). Run once in a container that mounts the reference:

    python tests/golden/make_lgf_golden.py /path/to/reference

The sample covers every entry with n1 <= 8, the table corners, and a seeded
random draw over the rest of 0 <= n3 <= n2 <= n1 <= 100.
"""
import json
import os
import random
import sys
import warnings


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IBLGF_REFERENCE")
    if not ref:
        sys.exit("usage: %s <reference tree> (or set IBLGF_REFERENCE)" % sys.argv[0])
    sys.path.insert(0, os.path.join(ref, "include/iblgf/lgf/lgf_table_gen"))
    import lgf_integrator  # noqa: E402

    entries = set()
    for n1 in range(0, 9):
        for n2 in range(0, n1 + 1):
            for n3 in range(0, n2 + 1):
                entries.add((n1, n2, n3))
    entries |= {(100, 0, 0), (100, 100, 0), (100, 100, 100), (100, 50, 25), (99, 98, 97)}
    rng = random.Random(20261203)
    while len(entries) < 1200:
        n1 = rng.randint(0, 100)
        n2 = rng.randint(0, n1)
        n3 = rng.randint(0, n2)
        entries.add((n1, n2, n3))
    out = []
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        for e in sorted(entries):
            out.append([e[0], e[1], e[2], float(lgf_integrator.lgf_int(*e))])
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "lgf_table_sample.json"), "w") as f:
        json.dump({"generator": "reference lgf_table_gen/lgf_integrator.py lgf_int (scipy quad, "
                                "epsabs 1e-16, epsrel 1e-15)",
                   "convention": "table value = integral (positive); LGF_GL_Lookup::get returns -value",
                   "entries": out}, f)


if __name__ == "__main__":
    main()
