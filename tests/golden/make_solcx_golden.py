"""Extract the SolCx verification values of the reference's own test suite
(tests/verification/linear/sol{c,k}x_*/{test.py,expected,more.opts} and the
options files they launch, src/models/analytics_vv/examples/*.opts) into
solcx_expected.json.  The solkx_* tests run the same model: it registers the
SolCx material geometry and error norms (src/models/analytics_vv/analytics_vv.c:
320-352, 414-416), with the SolCx parameters at their defaults.  Run in a
checkout that has the pTatin3d tree:

    python tests/golden/make_solcx_golden.py /path/to/pTatin3d

Each record keeps the mesh, the SolCx parameters, the component norms of the
initial residual (zero initial guess: the norm of the body-force right-hand
side per component) and the printed error norms
[inorms] h, ||v - v_ex||_L2, |E - E_ex|_H1s, H1, ||p - p_ex||_L2
(src/models/analytics_vv/analytics_vv.c:313-357), exactly as printed.
"""
import glob
import json
import os
import re
import sys

if len(sys.argv) < 2:
    sys.exit(f"usage: python {sys.argv[0]} <pTatin3d source tree>")
ref = sys.argv[1]


def options(path):
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0].strip()
        if line.startswith("-"):
            parts = line.split(None, 1)
            out[parts[0][1:]] = parts[1] if len(parts) > 1 else ""
    return out


out = {}
DEFAULTS = {"solcx_eta0": "1.0", "solcx_eta1": "1.0", "solcx_xc": "0.5", "solcx_n": "2"}  # analytics_vv.c:320-326
for d in sorted(glob.glob(os.path.join(ref, "tests/verification/linear/sol[ck]x_*"))):
    test = open(os.path.join(d, "test.py")).read()
    if re.search(r"ranks\s*=\s*1\b", test) is None:
        continue  # one-process runs only
    opts = dict(DEFAULTS)
    for f in re.findall(r"'(analytics-sol[ck]x-[a-z0-9]+\.opts)'", test):
        opts.update(options(os.path.join(ref, "src/models/analytics_vv/examples", f)))
    if os.path.exists(os.path.join(d, "more.opts")) and "more.opts" in test:
        opts.update(options(os.path.join(d, "more.opts")))
    text = open(os.path.join(d, "expected")).read()
    r0 = re.search(r"^\s*0 KSP Component U,V,W,P residual norm \[ (.*?) \]", text, re.M).group(1)
    inorms = re.search(r"^\[inorms\] (\S+)", text, re.M).group(1)
    out[os.path.basename(d)] = {
        "mx": int(opts["mx"]), "my": int(opts["my"]), "mz": int(opts["mz"]),
        "eta0": float(opts["solcx_eta0"]), "eta1": float(opts["solcx_eta1"]), "xc": float(opts["solcx_xc"]),
        "n": int(opts["solcx_n"]), "projection": int(opts["coefficient_projection_type"]),
        "r0_components": [s.strip() for s in r0.split(",")], "inorms": inorms.split(","),
        "source": os.path.relpath(os.path.join(d, "expected"), ref)}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "solcx_expected.json"), "w"), indent=1,
          sort_keys=True)
print(len(out), "records")
