"""Regenerate tests/golden/lqn_reference.json from UBOLT's own LQn generator.

Runs the reference's src/sn_lqn_table.py (it needs only mpmath) from a
checkout of stevendargaville/UBOLT and records, per order S2..S18, the level
cosines and the octant points with their weights exactly as that script
rounds them to double for its generated header. The library's own LQn
derivation is pinned against this file by tests/test_quadrature.py.

    python tests/golden/make_lqn_fixture.py /path/to/UBOLT
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_lqn_fixture.py /path/to/UBOLT")
ref = sys.argv[1]
sys.path.insert(0, os.path.join(ref, "src"))
import sn_lqn_table as gen  # noqa: E402

out = {}
for sn in range(2, 20, 2):
    o = gen.build_order(sn)
    gen.check_order(o)
    out[str(sn)] = {
        "mu": [float(v) for v in o["mu"]],
        "points": [[t[0], t[1], t[2], float(o["weights"][o["cls_of"][tuple(sorted(t))]])] for t in o["triples"]],
    }
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lqn_reference.json")
with open(path, "w") as fh:
    json.dump({"source": "stevendargaville/UBOLT src/sn_lqn_table.py build_order, rounded to double",
               "orders": out}, fh, indent=1)
print("wrote", path)
