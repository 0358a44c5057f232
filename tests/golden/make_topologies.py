"""Generates tests/golden/topologies.json by importing the reference's own pure-Python diagram
enumerator (python/triqs_xca/diag.py of TRIQS/xca), which needs only numpy.

Run where a checkout of the reference is available, giving its root directory:
    python tests/golden/make_topologies.py <path to the TRIQS/xca checkout>
"""
import importlib.util
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_topologies.py <path to the TRIQS/xca checkout>")
ref = sys.argv[1]
spec = importlib.util.spec_from_file_location("ref_diag", os.path.join(ref, "python", "triqs_xca", "diag.py"))
mod = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mod)
out = {}
for order in range(1, 5):
    out[str(order)] = {
        "connected": [[int(s), [list(map(int, p)) for p in t]] for s, t in mod.all_connected_pairings(order)],
        "all": [[int(s), [list(map(int, p)) for p in t]] for s, t in mod.all_pairings(order)],
    }
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "topologies.json"), "w") as f:
    json.dump(out, f, indent=0)
print({k: len(v["connected"]) for k, v in out.items()})
