"""Extract the initial Stokes residual of the reference's viscous-sinker
application tests (tests/application/linear/**/{opts,expected}) into
application_expected.json.  Run in a checkout that has the pTatin3d tree:

    python tests/golden/make_application_golden.py /path/to/pTatin3d

The outer Krylov solve starts from zero velocity and pressure
(ModelInitialCondition_ViscousSinker, src/models/viscous_sinker/
model_viscous_sinker_ops.c:1181-1220), so its first printed residual norm,
"0 KSP Residual norm", is the norm of the right-hand side: the body force of
the material points' density after their projection onto the Gauss points.
Each record keeps the mesh, the options the model reads and that value as
printed (6 significant digits), and the solver options and outcome: the outer
and inner relative tolerances, the Chebyshev degree of the smoother, the number
of multigrid levels, the per-level operator types (-A11_operator_type), the
printed outer residual history and the iteration count PETSc reports
("Linear solve converged due to CONVERGED_RTOL iterations N").
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
for opts_file in sorted(glob.glob(os.path.join(ref, "tests/application/linear/**/opts"), recursive=True)):
    d = os.path.dirname(opts_file)
    opts = {}
    for line in open(opts_file):
        line = line.split("#", 1)[0].strip()
        if line.startswith("-"):
            parts = line.split(None, 1)
            opts[parts[0][1:]] = parts[1] if len(parts) > 1 else ""
    if opts.get("ptatin_model") != "viscous_sinker":
        continue
    text = open(os.path.join(d, "expected")).read()
    m = re.search(r"^\s*0 KSP Residual norm (\S+)", text, re.M)
    # PETSc prints "%3D KSP Residual norm" after two spaces per tab level: the
    # outer solve at level 1, its inner solves at level 2
    outer = re.findall(r"^  (  \d| \d\d|\d\d\d) KSP Residual norm (\S+)", text, re.M)
    conv = re.search(r"Linear solve converged due to (\S+) iterations (\d+)", text)
    out[os.path.relpath(d, os.path.join(ref, "tests/application/linear"))] = {
        "mx": int(opts["mx"]), "my": int(opts["my"]), "mz": int(opts["mz"]),
        "eta0": float(opts.get("model_viscous_sinker_eta0", "1.0")),
        "eta1": float(opts.get("model_viscous_sinker_eta1", "1.0")),
        "rho0": float(opts.get("model_viscous_sinker_rho0", "0.0")),
        "rho1": float(opts.get("model_viscous_sinker_rho1", "1.0")),
        "lattice_layout_perturb": float(opts.get("lattice_layout_perturb", "0.1")),
        "projection": int(opts.get("coefficient_projection_type", "1")),
        "r0": m.group(1), "source": os.path.relpath(os.path.join(d, "expected"), ref),
        "ksp_rtol": float(opts.get("ksp_rtol", "1e-5")),
        "inner_rtol": float(opts.get("fieldsplit_u_ksp_rtol", "1e-5")),
        "cheb_its": int(opts.get("fieldsplit_u_mg_levels_ksp_max_it", "2")),
        "nlevels": int(opts.get("dau_nlevels", "1")),
        "a11_operator_type": opts.get("A11_operator_type", ""),
        "outer_history": [float(v) for _, v in outer],
        "outer_iterations": int(conv.group(2)) if conv else None,
        "converged_reason": conv.group(1) if conv else None}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "application_expected.json"), "w"),
          indent=1, sort_keys=True)
print(len(out), "records")
