"""Solve-level pin against the reference's own verification suite: the SolCx
analytic-solution tests (tests/verification/linear/solcx_*), whose printed
values tests/golden/make_solcx_golden.py extracted into solcx_expected.json.

* The initial residual's component norms (zero initial guess) are the norms
  of the body-force right-hand side; the oracle's assembly reproduces them.
* The oracle's discrete Stokes system [A11 A12; A21 0] with the reference's
  boundary convention, solved directly, gives a discrete solution whose error
  norms against the analytic solution -- computed by the reference's own
  Evaluate_uL2_symuH1_pL2 and SolCx code (oracle/_ref) -- equal the printed
  [inorms].  These norms depend on the discrete solution only, not on the
  solver that reached it (the reference solves to an absolute residual of
  1e-12).  The box is closed (free slip on every face), so the pressure is
  defined up to a constant; the printed pressure error is the one of the
  constant that minimises it, which the test takes too.
"""
import json
import os

import numpy as np
import pytest

from cases import solcx_case
from oracle.oracle import body_force, stokes_dense

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "solcx_expected.json")))


def rhs(restatement, case):
    bu = body_force(restatement, case["dims"], case["coords"], case["rho"], g=case["g"])
    bu[case["mask"].astype(bool)] = 0.0
    return bu


@pytest.mark.parametrize("name", sorted(GOLD))
def test_body_force_component_norms(restatement, name):
    rec = GOLD[name]
    case = solcx_case(rec["mx"], rec["my"], rec["mz"], rec["eta0"], rec["eta1"], rec["xc"], rec["n"])
    bu = rhs(restatement, case)
    got = [np.linalg.norm(bu[0::3]), np.linalg.norm(bu[1::3]), np.linalg.norm(bu[2::3]), 0.0]
    want = [float(v) for v in rec["r0_components"]]
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-12 * max(abs(w), 1e-30) + 1e-300, (name, got, want)


def solve_dense(restatement, case):
    """Direct solve of the oracle's Stokes system, one pressure dof held at 0
    (the closed box leaves the constant pressure free)."""
    dims, c = case["dims"], case["coords"]
    nel = dims[0] * dims[1] * dims[2]
    K = stokes_dense(restatement, dims, c, case["eta"], case["mask"])
    b = np.concatenate([rhs(restatement, case), np.zeros(4 * nel)])
    keep = np.ones(b.size, dtype=bool)
    keep[c.size] = False
    x = np.zeros(b.size)
    x[keep] = np.linalg.solve(K[np.ix_(keep, keep)], b[keep])
    assert np.linalg.norm(K @ x - b) <= 1e-12 * np.linalg.norm(b)
    return x[:c.size], x[c.size:]


def pressure_fitted_norms(reference_kernels, prm, u, p):
    """Error norms with the free constant pressure set to minimise the pressure
    error: the constant mode is the first P1disc basis function of every
    element, and ||p_h + s - p_ex||^2 is quadratic in s, so three evaluations
    give its minimum."""
    def norms(shift):
        q = np.array(p, dtype=np.float64).copy()
        q[0::4] += shift
        return reference_kernels.solcx_norms(*prm, u, q)
    f0, f1, fm = norms(0.0)[3] ** 2, norms(1.0)[3] ** 2, norms(-1.0)[3] ** 2
    return norms(-(f1 - fm) / 2.0 / (f1 + fm - 2.0 * f0))


@pytest.mark.parametrize("name", sorted(n for n in GOLD if GOLD[n]["mx"] * GOLD[n]["my"] * GOLD[n]["mz"] <= 72))
def test_discrete_solution_reproduces_reference_error_norms(restatement, reference_kernels, name):
    rec = GOLD[name]
    prm = (rec["eta0"], rec["eta1"], rec["xc"], rec["n"])
    case = solcx_case(rec["mx"], rec["my"], rec["mz"], *prm)
    u, p = solve_dense(restatement, case)
    reference_kernels.setup(case["dims"], case["coords"], case["eta"].reshape(-1))
    got = pressure_fitted_norms(reference_kernels, prm, u, p)
    want = [float(v) for v in rec["inorms"]]
    assert abs(want[0] - 1.0 / rec["mx"]) <= 1e-12
    for g, w in zip(got, want[1:]):
        assert abs(g - w) <= 1e-8 * abs(w), (name, got, want)


@pytest.mark.parametrize("name", sorted(GOLD))
def test_cpu_solver_reproduces_reference_error_norms(reference_kernels, name):
    """The solver restated on the host (the device solver's algorithm: FGMRES,
    Schur upper, Galerkin multigrid with Chebyshev/Jacobi) on every SolCx case,
    12x12x2 included, solved to 1e-11: the reference's printed norms."""
    from oracle.cpu_solver import CpuStokesSolver
    rec = GOLD[name]
    prm = (rec["eta0"], rec["eta1"], rec["xc"], rec["n"])
    case = solcx_case(rec["mx"], rec["my"], rec["mz"], *prm)
    S = CpuStokesSolver(case["dims"], case["coords"], case["eta"], case["rho"], case["bits"], nlevels=2, g=case["g"])
    u, p, its, rt, _ = S.solve(rtol=1e-11, max_it=500)
    assert rt <= 1e-11
    reference_kernels.setup(case["dims"], case["coords"], case["eta"].reshape(-1))
    got = pressure_fitted_norms(reference_kernels, prm, u, p)
    want = [float(v) for v in rec["inorms"][1:]]
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-8 * abs(w), (name, got, want)
