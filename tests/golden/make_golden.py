"""Extract the operator known-answer values from the reference's own test
fixtures (tests/integration/operator/**/{opts,expected}) into
reference_expected.json.  Run in a checkout that has the pTatin3d tree:

    python tests/golden/make_golden.py /path/to/pTatin3d

Each record keeps the mesh size, the sinker viscosity option and the printed
y.y = ||y||^2 of every operator test, exactly as printed (9 digits).
"""
import glob
import json
import os
import re
import sys

if len(sys.argv) < 2:
    sys.exit(f"usage: python {sys.argv[0]} <pTatin3d source tree>")
ref = sys.argv[1]
out = {}
for exp in sorted(glob.glob(os.path.join(ref, "tests/integration/operator/**/expected"), recursive=True)):
    d = os.path.dirname(exp)
    opts = open(os.path.join(d, "opts")).read()
    opt = lambda k, dflt=None: (re.search(rf"^-{k}\s+(\S+)", opts, re.M) or [None, dflt])[1]
    if "-compare_operators" not in opts:
        continue
    text = open(exp).read()
    rec = {"mx": int(opt("mx")), "my": int(opt("my")), "mz": int(opt("mz")),
           "eta1": float(opt("model_viscous_sinker_eta1", "1.0")), "a11_op": opt("a11_op", "default"),
           "source": os.path.relpath(exp, ref)}
    for test in ("A11", "A21", "A12", "A", "diagA11"):
        m = re.search(rf"Test \[compare_mf_{test}\].*?\n\s+y\.y\s+=\s+(\S+)", text, re.S)
        if m:
            rec[test] = m.group(1)
    out[os.path.relpath(d, os.path.join(ref, "tests/integration/operator"))] = rec
json.dump(out, open(os.path.join(os.path.dirname(__file__), "reference_expected.json"), "w"), indent=1, sort_keys=True)
print(len(out), "records")
