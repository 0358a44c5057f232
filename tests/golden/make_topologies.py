"""Generates tests/golden/topologies.json by importing the reference's own pure-Python diagram
enumerator (python/triqs_xca/diag.py of TRIQS/xca), which needs only numpy.

Run in the build container, where the reference is mounted:
    python tests/golden/make_topologies.py /root/reference
"""
import importlib.util
import json
import os
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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
