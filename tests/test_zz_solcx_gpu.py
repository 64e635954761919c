"""The device solver (p3d_solver_*) on the reference's SolCx verification
tests (tests/verification/linear/solcx_*): solved to a relative residual of
1e-11, its velocity, strain-rate and pressure error norms against the analytic
solution -- computed by the reference's own Evaluate_uL2_symuH1_pL2 and SolCx
code (oracle/_ref) -- equal the values the reference printed, as the host
restatement of the same solver's do (tests/test_solcx_verification.py).
Collected last (file name) so a failure here does not hide the rest of the
suite.
"""
import json
import os

import numpy as np
import pytest

from cases import solcx_case

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "solcx_expected.json")))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_device_solver_reproduces_reference_error_norms(cuda, reference_kernels, name):
    from ptatin3d_b200.solver import StokesSolver
    from test_solcx_verification import pressure_fitted_norms
    rec = GOLD[name]
    prm = (rec["eta0"], rec["eta1"], rec["xc"], rec["n"])
    case = solcx_case(rec["mx"], rec["my"], rec["mz"], *prm)
    S = StokesSolver(*case["dims"], case["bits"], nlevels=2, rtol=1e-11, max_it=500)
    S.setup(case["coords"], case["eta"])
    S.set_rhs_body_force(case["rho"], g=case["g"])
    u, p, st = S.solve(raise_on_noconv=False)
    S.destroy()
    assert st["converged"] and st["rfinal"] <= 1e-11 * st["r0"], st
    reference_kernels.setup(case["dims"], case["coords"], case["eta"].reshape(-1))
    got = pressure_fitted_norms(reference_kernels, prm, u.cpu().numpy(), p.cpu().numpy())
    want = [float(v) for v in rec["inorms"][1:]]
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-7 * abs(w), (name, got, want)
    assert np.isfinite(got).all()
