"""The device path against values the reference's own test suite prints.

* Operator tests with the eta1 = 10 viscous sinker
  (tests/integration/operator/**/expected): the markers go through the device
  Q1 projection (p3d_marker_project) into the device operator, whose A11 and
  diag(A11) y.y equal the printed values.
* Viscous-sinker application tests (tests/application/linear/**/expected):
  the first printed residual, from zero velocity and pressure, is the norm of
  the body force; the device projection of the markers' density and the
  device residual (p3d_stokes_residual) reproduce it.
* SolCx verification tests (tests/verification/linear/sol{c,k}x_*): the
  device solver (p3d_solver_*), solved to a relative residual of 1e-11, gives
  velocity, strain-rate and pressure error norms against the analytic
  solution -- computed by the reference's own Evaluate_uL2_symuH1_pL2 and
  SolCx code (oracle/_ref) -- equal to the printed ones, as the host
  restatement of the same solver does (tests/test_solcx_verification.py).

Collected last (file name) so a failure here does not hide the rest of the
suite.
"""
import json
import os

import numpy as np
import pytest

from cases import bump_case, sinker_markers, solcx_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "solcx_expected.json")))
OPS = json.load(open(os.path.join(HERE, "golden", "reference_expected.json")))
APP = json.load(open(os.path.join(HERE, "golden", "application_expected.json")))


def _device(cuda, a, dt):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)


@pytest.mark.parametrize("name", sorted(APP))
def test_device_rhs_matches_reference_application(cuda, name):
    import torch

    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    from ptatin3d_b200.operators import MatStokesMF, mesh_desc_whole
    rec = APP[name]
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    eta_q, rho_q = update_gauss_properties(case["dims"], PROJ_Q1, _device(cuda, wil, torch.int32),
                                           _device(cuda, xi, torch.float64), _device(cuda, eta_p, torch.float64),
                                           _device(cuda, rho_p, torch.float64))
    op = MatStokesMF(mesh_desc_whole(*case["dims"], case["bits"]))
    op.set_coefficients(_device(cuda, case["coords"], torch.float64), eta_q)
    fu = torch.zeros(rho_q.shape[0], 27, 3, dtype=torch.float64, device=cuda)
    fu[..., 1] = rho_q  # gravity (0, 1, 0), the reference's default (src/ptatin3d.c:94-104)
    u = torch.zeros(op.n_velocity, dtype=torch.float64, device=cuda)
    p = torch.zeros(op.n_pressure, dtype=torch.float64, device=cuda)
    ru, rp = op.residual(u, p, fu=fu)
    val = float(torch.sqrt(ru @ ru + rp @ rp))
    gold = float(rec["r0"])
    assert abs(val - gold) <= 5e-6 * gold, (name, val, gold)


@pytest.mark.parametrize("name", sorted(n for n, r in OPS.items() if r["eta1"] != 1.0))
def test_device_projection_and_operator_match_reference_expected(cuda, name):
    import torch

    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    from ptatin3d_b200.operators import MatStokesMF, mesh_desc_whole
    rec = OPS[name]
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, eta1=rec["eta1"])
    t = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)
    eta_q, _ = update_gauss_properties(case["dims"], PROJ_Q1, t(wil, torch.int32), t(xi, torch.float64),
                                       t(eta_p, torch.float64), t(rho_p, torch.float64))
    op = MatStokesMF(mesh_desc_whole(*case["dims"], case["bits"]))
    op.set_coefficients(t(case["coords"], torch.float64), eta_q)
    x = t(case["x"], torch.float64)
    y = torch.empty_like(x)
    op.mult(x, y)
    d = torch.empty_like(x)
    op.get_diagonal(d)
    for val, key in ((float(y @ y), "A11"), (float(d @ d), "diagA11")):
        gold = float(rec[key])
        assert abs(val - gold) <= 5e-9 * abs(gold), (name, key, val, gold)


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


def test_device_marker_hierarchy_levels_match_oracle(cuda, restatement):
    """The reference's projection type 1 end to end on the device: markers ->
    Q1 projection -> the nodal viscosity feeds the solver's Q1 coefficient
    hierarchy (p3d_solver_setup_nodal); every level operator equals the
    oracle's MatMult with the restated hierarchy started from the same nodal
    field (src/material_point_utils.c:1267-1420)."""
    import torch

    from oracle.oracle import marker_project, matmult_a11
    from ptatin3d_b200 import COARSE_ETA_Q1, COARSE_REDISC
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    from ptatin3d_b200.solver import StokesSolver
    m, nlev = 8, 3
    case = bump_case(m, m, m)
    wil, xi, eta_p, rho_p = sinker_markers(case, eta0=1.0, eta1=100.0)
    eta_q, _, v = update_gauss_properties(case["dims"], PROJ_Q1, _device(cuda, wil, torch.int32),
                                          _device(cuda, xi, torch.float64), _device(cuda, eta_p, torch.float64),
                                          _device(cuda, rho_p, torch.float64), nodal=True)
    bits = M.FREE_SLIP
    S = StokesSolver(m, m, m, bits, nlevels=nlev, coarse_op=COARSE_REDISC, coarse_eta=COARSE_ETA_Q1)
    S.setup(case["coords"], eta_q, eta_nodes=v)
    e_ref, _, v_ref = marker_project(case["dims"], 1, wil, xi, eta_p, rho_p, nodal=True)
    etas = restatement.eta_hierarchy_from_nodes(case["dims"], e_ref, v_ref, nlev)
    rng = np.random.default_rng(6)
    cl = np.asarray(case["coords"])
    for depth in range(nlev):
        mm = m >> depth
        if depth:
            nf = 2 * (2 * mm) + 1
            cl = cl.reshape(nf, nf, nf, 3)[::2, ::2, ::2].reshape(-1).copy()  # injection
        x = rng.uniform(-1, 1, size=3 * (2 * mm + 1) ** 3)
        y = S.level_apply(nlev - 1 - depth, x).cpu().numpy()
        mask = M.dirichlet_mask(mm, mm, mm, bits)
        ref = matmult_a11(lambda w: restatement.a11_raw((mm, mm, mm), cl, etas[depth], w), x, mask)
        assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref), depth
    S.destroy()


def test_device_solver_takes_the_reference_application_iteration_count(cuda):
    """The viscous-sinker application solve with the reference's own solver
    options (tests/application/linear/sinker_galerkin_8x8x8/opts: 3 levels,
    Galerkin coarse operators, Chebyshev(10)/Jacobi, inner velocity solve to
    rtol 1e-2, outer FGMRES to rtol 1e-3), from the device projection of the
    markers: the reference converges in 17 outer iterations; the device solve
    (inner conjugate gradients in a conditional graph loop, exact 4x4 Schur
    blocks) takes that count to within 3 and starts from the printed residual."""
    import torch

    from ptatin3d_b200 import SCHUR_ETA_QP
    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    from ptatin3d_b200.solver import StokesSolver
    rec = APP["sinker_galerkin_8x8x8"]
    assert rec["a11_operator_type"] == "2,2,0" and rec["outer_iterations"] == 17
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    eta_q, rho_q = update_gauss_properties(case["dims"], PROJ_Q1, _device(cuda, wil, torch.int32),
                                           _device(cuda, xi, torch.float64), _device(cuda, eta_p, torch.float64),
                                           _device(cuda, rho_p, torch.float64))
    S = StokesSolver(*case["dims"], case["bits"], nlevels=rec["nlevels"], cheb_its=rec["cheb_its"],
                     rtol=rec["ksp_rtol"], max_it=100, inner_rtol=rec["inner_rtol"], inner_its=200,
                     schur_eta=SCHUR_ETA_QP)
    S.setup(_device(cuda, case["coords"], torch.float64), eta_q)
    S.set_rhs_body_force(rho_q, (0.0, 1.0, 0.0))
    _, _, st = S.solve()
    S.destroy()
    assert st["converged"]
    assert abs(st["r0"] - rec["outer_history"][0]) <= 5e-6 * rec["outer_history"][0]
    assert abs(st["iterations"] - rec["outer_iterations"]) <= 3, st
    assert st["iterations"] <= st["inner_iterations"] <= 4 * st["iterations"]
