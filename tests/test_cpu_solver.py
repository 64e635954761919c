"""The CPU restatement of the solver (oracle/cpu_solver.py, the CPU solve
baseline of bench.py) solves the oracle's assembled Stokes system, and on the
GPU it takes the same path as the device solver."""
import os

import numpy as np
import pytest

from cases import rel
from oracle.oracle import body_force, stokes_dense
from ptatin3d_b200 import mesh as M

BITS = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)


def sinker(m, contrast, seed=1):
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(4, seed, 0.15)
    return c, M.sinker_eta(qp, cen, r, 1.0, contrast), M.sinker_density(qp, cen, r, 1.0, 1.01)


def test_lattice_mask_matches_mesh_helper():
    from oracle.cpu_solver import lattice_mask
    for dims, bits in (((3, 4, 5), BITS), ((2, 2, 2), M.FREE_SLIP)):
        n = tuple(2 * d + 1 for d in dims)
        assert np.array_equal(lattice_mask(n, bits), M.dirichlet_mask(*dims, bits).astype(bool))


def test_cpu_solver_solves_assembled_system(restatement, reference_kernels):
    from oracle.cpu_solver import CpuStokesSolver
    m = 4
    c, eta, rho = sinker(m, 1e2)
    S = CpuStokesSolver(m, c, eta, rho, BITS, nlevels=2, schur_geomean=False)
    u, p, its, rt, _ = S.solve(rtol=1e-11, max_it=400)
    assert rt <= 1e-10
    mask = M.dirichlet_mask(m, m, m, BITS)
    K = stokes_dense(restatement, (m, m, m), c, eta, mask)
    bu = body_force(restatement, (m, m, m), c, rho)
    bu[mask.astype(bool)] = 0.0
    b = np.concatenate([bu, np.zeros(4 * m ** 3)])
    x = np.concatenate([u, p])
    assert np.linalg.norm(K @ x - b) <= 1e-9 * np.linalg.norm(b)


@pytest.mark.gpu
def test_cpu_and_gpu_solvers_agree(cuda, reference_kernels):
    """Same algorithm on both sides: iteration counts within 15 %, solutions
    equal to the tolerance the solves were run to."""
    from oracle.cpu_solver import CpuStokesSolver
    from ptatin3d_b200 import SCHUR_ETA_GEOMEAN
    from ptatin3d_b200.solver import StokesSolver
    m = 8
    c, eta, rho = sinker(m, 1e3)
    C = CpuStokesSolver(m, c, eta, rho, BITS, nlevels=3)
    uc, pc, itc, rtc, _ = C.solve(rtol=1e-9, max_it=2000)
    G = StokesSolver(m, m, m, BITS, nlevels=3, rtol=1e-9, max_it=2000, schur_eta=SCHUR_ETA_GEOMEAN)
    G.setup(c, eta)
    G.set_rhs_body_force(rho)
    ug, pg, st = G.solve()
    assert rtc <= 1e-9 and st["converged"]
    assert abs(st["iterations"] - itc) <= 0.15 * itc + 3
    assert rel(ug.cpu().numpy(), uc) <= 1e-6


def test_slab_partitioned_reference_apply(reference_kernels):
    """The slab layout of the CPU baseline computes the same MatMult as the
    whole-mesh reference kernel (partial sums added on the shared planes)."""
    from oracle.cpu_slabs import slab_apply_time
    m = 6
    c = M.perturb_interior(M.uniform_coords(m, m, m), m, m, m, frac=0.2, seed=2)
    eta = 10 ** np.random.default_rng(1).uniform(-1, 1, size=(m ** 3, 27))
    x = np.random.default_rng(2).uniform(-1, 1, size=c.size)
    t, y = slab_apply_time(c, eta, x, m, 3, steps=1, warmup=0, collect=True)
    assert t > 0.0
    reference_kernels.setup((m, m, m), c, eta)
    assert rel(y, reference_kernels.a11_raw(x, "avx")) <= 1e-12


def _application_case(name):
    import json

    from cases import bump_case, sinker_markers
    from oracle.oracle import marker_project
    rec = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                      "application_expected.json")))[name]
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    eta_q, rho_q = marker_project(case["dims"], 1, wil, xi, eta_p, rho_p)
    return rec, case, eta_q, rho_q


def test_restatement_takes_the_reference_application_iteration_count(reference_kernels):
    """The reference's viscous-sinker solve with its own solver options
    (tests/application/linear/sinker_galerkin_8x8x8/opts: 3 levels, Galerkin
    coarse operators, Chebyshev(10)/Jacobi, inner velocity solve to rtol 1e-2,
    outer FGMRES to rtol 1e-3) converges in 17 outer iterations.  The host
    restatement of the device solver (inner conjugate gradients instead of
    FGMRES, exact 4x4 Schur blocks instead of their Jacobi diagonal) takes
    that count to within 3 iterations.  PETSc is not vendored, so the count is
    compared, not the history."""
    from oracle.cpu_solver import CpuStokesSolver
    rec, case, eta_q, rho_q = _application_case("sinker_galerkin_8x8x8")
    assert rec["a11_operator_type"] == "2,2,0" and rec["outer_iterations"] == 17
    S = CpuStokesSolver(case["dims"], case["coords"], eta_q, rho_q, case["bits"], nlevels=rec["nlevels"],
                        cheb_its=rec["cheb_its"], schur_geomean=False, g=(0.0, 1.0, 0.0),
                        inner_rtol=rec["inner_rtol"], inner_its=200)
    _, _, its, rt, _ = S.solve(rtol=rec["ksp_rtol"], max_it=100)
    assert rt <= rec["ksp_rtol"]
    assert abs(its - rec["outer_iterations"]) <= 3, its
    assert its <= S.inner_total <= 4 * its  # a few inner iterations per outer one, as the reference prints


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [64, 32])
def test_cpu_and_gpu_inner_solves_agree(cuda, reference_kernels, prec):
    """With the velocity block solved to a relative tolerance by inner
    conjugate gradients, the device solve (FP64, or FP32 multigrid) and the
    host restatement (both estimate lambda_max from the same start vector)
    take outer and total inner iteration counts within 25 % of each other
    (35 % for the FP32 multigrid against the FP64 restatement) and reach the
    same solution."""
    from oracle.cpu_solver import CpuStokesSolver
    from ptatin3d_b200 import SCHUR_ETA_GEOMEAN
    from ptatin3d_b200.solver import StokesSolver
    m = 8
    c, eta, rho = sinker(m, 1e3)
    C = CpuStokesSolver(m, c, eta, rho, BITS, nlevels=3, inner_rtol=1e-2, inner_its=100)
    uc, pc, itc, rtc, _ = C.solve(rtol=1e-9, max_it=500)
    G = StokesSolver(m, m, m, BITS, nlevels=3, rtol=1e-9, max_it=500, schur_eta=SCHUR_ETA_GEOMEAN,
                     inner_rtol=1e-2, inner_its=100, mg_precision=prec)
    G.setup(c, eta)
    G.set_rhs_body_force(rho)
    ug, pg, st = G.solve()
    assert rtc <= 1e-9 and st["converged"]
    assert abs(st["lmax_fine"] / C.lv[-1].lmax - 1.0) <= 1e-8  # the same Lanczos start vector
    # the restatement runs its multigrid in FP64; against the device's FP32
    # multigrid the variable inner solves take different paths.  Even in FP64
    # the rounding order of the device sums (and its single Gram-Schmidt pass
    # where the projection removed little) steers the 1e-2 inner solves of a
    # contrast-1e3 solve to rtol 1e-9 apart over some hundred outer
    # iterations: measured 133 against 166 outer iterations, and inner totals
    # 16 % apart, depending on the device's reduction order.
    tol, tol_in = (0.25, 0.25) if prec == 64 else (0.35, 0.35)
    assert abs(st["iterations"] - itc) <= tol * itc + 2, (st["iterations"], itc)
    assert abs(st["inner_iterations"] - C.inner_total) <= tol_in * C.inner_total + 3, (st, itc, C.inner_total)
    assert st["inner_iterations"] > st["iterations"]
    # a variable (inner-tolerance) preconditioner: both stop at rtol 1e-9 on
    # different Krylov paths, so their solutions differ by the conditioning
    assert rel(ug.cpu().numpy(), uc) <= 2e-5
