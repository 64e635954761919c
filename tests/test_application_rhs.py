"""The first residual the reference's viscous-sinker application tests print
(tests/application/linear/**/expected, extracted into
tests/golden/application_expected.json): from zero velocity and pressure it is
the norm of the right-hand side, the body force of the material points'
density projected onto the Gauss points.  Reproducing it pins the marker
lattice, the Q1 projection (type 1, the default), the default gravity
(0, 1, 0) (src/ptatin3d.c:94-104), the body-force assembly and the
free-slip / free-surface Dirichlet rows together; printed to 6 digits."""
import json
import os

import numpy as np
import pytest

from cases import bump_case, sinker_markers
from oracle.oracle import body_force, marker_project

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "application_expected.json")))
GRAVITY = (0.0, 1.0, 0.0)


def rhs_norm(restatement, case, rho_q):
    bu = body_force(restatement, case["dims"], case["coords"], rho_q, g=GRAVITY)
    bu[case["mask"].astype(bool)] = 0.0
    return float(np.linalg.norm(bu))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_restatement_rhs_matches_reference_application(restatement, name):
    rec = GOLD[name]
    assert rec["lattice_layout_perturb"] == 0.0 and rec["projection"] == 1
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    _, rho_q = marker_project(case["dims"], 1, wil, xi, eta_p, rho_p)
    gold = float(rec["r0"])
    assert abs(rhs_norm(restatement, case, rho_q) - gold) <= 5e-6 * gold


@pytest.mark.parametrize("name", sorted(GOLD))
def test_reference_projection_rhs_matches_reference_application(restatement, reference_kernels, name):
    """The same with the reference's own compiled projection."""
    rec = GOLD[name]
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    nel = rec["mx"] * rec["my"] * rec["mz"]
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    reference_kernels.setup(case["dims"], case["coords"], np.ones(27 * nel))
    _, rho_q = reference_kernels.marker_project(1, wil, xi, eta_p, rho_p)
    gold = float(rec["r0"])
    assert abs(rhs_norm(restatement, case, rho_q) - gold) <= 5e-6 * gold
