"""GPU Stokes solve (FGMRES + Schur upper + GMG) against the CPU oracle.

The oracle solve assembles [A11 A12; A21 0] by probing the CPU restatement's
operators and solves it densely (small meshes).  Solver-level PETSc parity is
not available (PETSc is not vendored), so the solve is checked against this
exact discrete solution instead.
"""
import numpy as np
import pytest
import torch

from cases import rel
from oracle.oracle import body_force, matmult_a11, stokes_dense, stokes_dense_solve
from ptatin3d_b200 import (COARSE_GALERKIN, COARSE_REDISC, PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN, SCHUR_ETA_QP,
                           P3DError)
from ptatin3d_b200 import mesh as M
from ptatin3d_b200.solver import StokesSolver

pytestmark = pytest.mark.gpu

# free slip on the walls and the base, free surface on top (z max)
BITS = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)


def sinker(m, nsph=2, radius=0.2, contrast=1e2, seed=1, deform=0.0):
    c = M.uniform_coords(m, m, m)
    if deform:
        c = M.perturb_interior(c, m, m, m, frac=deform, seed=seed)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(nsph, seed, radius)
    eta = M.sinker_eta(qp, cen, r, 1.0, contrast)
    rho = M.sinker_density(qp, cen, r, 1.0, 1.01)
    return c, eta, rho


@pytest.mark.parametrize("deform", [0.0, 0.1])
def test_solve_matches_dense_oracle(cuda, restatement, deform):
    m = 4
    c, eta, rho = sinker(m, deform=deform)
    mask = M.dirichlet_mask(m, m, m, BITS)
    bu = body_force(restatement, (m, m, m), c, rho)
    bu[mask.astype(bool)] = 0.0
    K = stokes_dense(restatement, (m, m, m), c, eta, mask)
    b = np.concatenate([bu, np.zeros(4 * m ** 3)])
    xref = np.linalg.solve(K, b)
    u_ref, p_ref = xref[:bu.size], xref[bu.size:]
    S = StokesSolver(m, m, m, BITS, nlevels=2, rtol=1e-11, max_it=300)
    S.setup(c, eta)
    S.set_rhs_body_force(rho, (0.0, 0.0, -1.0))
    u, p, st = S.solve()
    assert st["converged"]
    xg = np.concatenate([u.cpu().numpy(), p.cpu().numpy()])
    # the GPU solution solves the oracle's assembled system to the requested tolerance
    assert np.linalg.norm(K @ xg - b) <= 1e-10 * np.linalg.norm(b)
    # and agrees with its direct solution to within the system's conditioning
    assert rel(xg[:bu.size], u_ref) <= 1e-6
    assert rel(xg[bu.size:], p_ref) <= 1e-6


def test_rhs_matches_oracle(cuda, restatement):
    m = 6
    c, eta, rho = sinker(m, deform=0.1)
    bu_ref = body_force(restatement, (m, m, m), c, rho, (0.3, -0.2, -1.0))
    bu_ref[M.dirichlet_mask(m, m, m, BITS).astype(bool)] = 0.0
    sols = []
    for use_kernel in (True, False):
        S = StokesSolver(m, m, m, BITS, nlevels=2, rtol=1e-11, max_it=300)
        S.setup(c, eta)
        if use_kernel:
            S.set_rhs_body_force(rho, (0.3, -0.2, -1.0))
        else:
            S.set_rhs(bu_ref, np.zeros(S.np))
        sols.append(S.solve()[0].cpu().numpy())
    assert rel(sols[0], sols[1]) <= 1e-9


@pytest.mark.parametrize("prec", [PREC_F64, PREC_F32])
def test_multilevel_solve_converges(cuda, prec):
    """3-level Galerkin GMG, viscosity contrast 1e2: the iteration count of the
    FP64 and the mixed-precision preconditioner are the same (FP32 smoothing
    does not slow the outer FP64 iteration down)."""
    m = 16
    c, eta, rho = sinker(m, nsph=4, radius=0.12, contrast=1e2)
    S = StokesSolver(m, m, m, BITS, nlevels=3, rtol=1e-6, mg_precision=prec)
    S.setup(c, eta)
    S.set_rhs_body_force(rho)
    u, p, st = S.solve()
    assert st["converged"] and st["iterations"] <= 60
    assert st["rfinal"] <= 1.0000001e-6 * st["r0"]


def test_high_contrast_solve_converges(cuda):
    """Contrast 1e3 with the inner velocity CG and the geometric-mean Schur weighting."""
    m = 16
    c, eta, rho = sinker(m, nsph=4, radius=0.12, contrast=1e3)
    S = StokesSolver(m, m, m, BITS, nlevels=3, rtol=1e-6, max_it=400, inner_its=3, schur_eta=SCHUR_ETA_GEOMEAN,
                     mg_precision=PREC_F32)
    S.setup(c, eta)
    S.set_rhs_body_force(rho)
    u, p, st = S.solve()
    assert st["converged"] and st["iterations"] <= 200


def test_redisc_coarse_levels_still_supported(cuda):
    m = 8
    c, eta, rho = sinker(m, contrast=10.0)
    S = StokesSolver(m, m, m, BITS, nlevels=3, coarse_op=COARSE_REDISC, rtol=1e-8)
    S.setup(c, eta)
    S.set_rhs_body_force(rho)
    assert S.solve()[2]["converged"]


def test_mixed_precision_error_vs_fp64_oracle_solve(cuda):
    """The outer FP64 FGMRES recovers full accuracy from the FP32 V-cycle: the
    mixed-precision solution agrees with a tightly converged FP64 solve."""
    m = 16
    c, eta, rho = sinker(m, nsph=4, radius=0.12, contrast=1e3)
    kw = dict(nlevels=3, inner_its=3, schur_eta=SCHUR_ETA_GEOMEAN, max_it=1500)
    ref = StokesSolver(m, m, m, BITS, rtol=1e-11, **kw)
    ref.setup(c, eta)
    ref.set_rhs_body_force(rho)
    u64, p64, _ = ref.solve()
    mix = StokesSolver(m, m, m, BITS, rtol=1e-9, mg_precision=PREC_F32, **kw)
    mix.setup(c, eta)
    mix.set_rhs_body_force(rho)
    u32, p32, st = mix.solve()
    assert st["converged"]
    assert rel(u32.cpu().numpy(), u64.cpu().numpy()) <= 1e-6
    assert rel(p32.cpu().numpy(), p64.cpu().numpy()) <= 1e-5


def test_mixed_precision_at_rtol_1e6_on_the_sinker_solve(cuda):
    """The 32^3 sinker solve (8 spheres of radius 0.1, viscosity contrast 1e4,
    density +1 %, 4 Galerkin levels) at rtol 1e-6, in FP64 and with the FP32
    multigrid, against an FP64 solve to rtol 1e-10 (the FP64 oracle solve).
    At this tolerance both solutions carry the iteration error of rtol 1e-6
    on an ill-conditioned system (about 1e-4 relative); the mixed-precision
    solution lies no farther from the oracle than the FP64 one, so the FP32
    smoother adds no error of its own.  The mixed-minus-FP64 difference is
    the difference of two rtol-1e-6 iterates (5e-6 to 1.3e-5 measured), not
    rounding."""
    m = 32
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(8, 1, 0.1)
    eta, rho = M.sinker_eta(qp, cen, r, 1.0, 1e4), M.sinker_density(qp, cen, r, 1.0, 1.01)
    sol = {}
    for name, prec, rtol in (("oracle", PREC_F64, 1e-10), ("fp64", PREC_F64, 1e-6), ("mixed", PREC_F32, 1e-6)):
        S = StokesSolver(m, m, m, BITS, nlevels=4, rtol=rtol, max_it=8000, mg_precision=prec,
                         schur_eta=SCHUR_ETA_GEOMEAN)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        u, p, st = S.solve()
        assert st["converged"], name
        sol[name] = (u.cpu().numpy(), p.cpu().numpy())
        S.destroy()
    (uo, po), (u64, p64), (u32, p32) = sol["oracle"], sol["fp64"], sol["mixed"]
    e64, e32 = rel(u64, uo), rel(u32, uo)
    print(f"velocity error vs the FP64 oracle solve: FP64 {e64:.2e}, mixed {e32:.2e}; "
          f"mixed - FP64 {rel(u32, u64):.2e}; pressure: FP64 {rel(p64, po):.2e}, mixed {rel(p32, po):.2e}")
    assert e64 <= 1e-3 and e32 <= 1e-3
    assert e32 <= 1.5 * e64  # FP32 smoothing adds nothing beyond the rtol-1e-6 iteration error
    assert rel(u32, u64) <= 5e-5


def galerkin_oracle(R, m, c, eta, nlev):
    """Level operators of the Galerkin hierarchy from the oracle's fine MatMult:
    A_{l-1} = P~^T A_l P~ + I on Dirichlet dofs, P~ the masked trilinear prolongation."""
    fine_mask = M.dirichlet_mask(m, m, m, BITS)
    ops = [lambda v: matmult_a11(lambda w: R.a11_raw((m, m, m), c, eta.reshape(-1), w), v, fine_mask)]
    masks = [fine_mask.astype(bool)]
    mm = m
    for _ in range(nlev - 1):
        mm //= 2
        cm = M.dirichlet_mask(mm, mm, mm, BITS).astype(bool)
        fm, A, cn = masks[-1], ops[-1], (2 * mm + 1,) * 3

        def Ac(v, fm=fm, A=A, cm=cm, cn=cn):
            xf = R.prolong(cn, 3, np.where(cm, 0.0, v))
            xf[fm] = 0.0
            yf = A(xf)
            yf[fm] = 0.0
            y = R.restrict(cn, 3, yf)
            y[cm] = v[cm]
            return y
        ops.append(Ac)
        masks.append(cm)
    return ops[::-1]  # coarsest first


def test_galerkin_levels_match_oracle(cuda, restatement):
    m, nlev = 8, 3
    c, eta, _ = sinker(m, contrast=1e3, deform=0.1)
    S = StokesSolver(m, m, m, BITS, nlevels=nlev, coarse_op=COARSE_GALERKIN)
    S.setup(c, eta)
    ops = galerkin_oracle(restatement, m, c, eta, nlev)
    rng = np.random.default_rng(3)
    for lvl in range(nlev):
        mm = m >> (nlev - 1 - lvl)
        x = rng.uniform(-1, 1, size=3 * (2 * mm + 1) ** 3)
        y = S.level_apply(lvl, x).cpu().numpy()
        assert rel(y, ops[lvl](x)) <= 1e-12, lvl


@pytest.mark.parametrize("weighting", [SCHUR_ETA_QP, SCHUR_ETA_GEOMEAN])
def test_schur_blocks_match_oracle(cuda, restatement, weighting):
    """zp = S~^{-1} rp of the block preconditioner against the oracle's
    viscosity-scaled pressure mass matrix (src/stokes_assembly.c:299-450)."""
    m = 6
    c, eta, _ = sinker(m, contrast=1e3, deform=0.15)
    S = StokesSolver(m, m, m, BITS, nlevels=2, schur_eta=weighting)
    S.setup(c, eta)
    e = eta.reshape(-1, 27)
    if weighting == SCHUR_ETA_GEOMEAN:
        e = np.repeat(np.exp(np.log(e).mean(axis=1, keepdims=True)), 27, axis=1)
    blocks = restatement.schur_mass((m, m, m), c, e.reshape(-1))
    rp = np.random.default_rng(2).standard_normal(S.np)
    _, zp = S.apply_pc(np.zeros(S.nu), rp)
    ref = np.linalg.solve(blocks, rp.reshape(-1, 4, 1)).reshape(-1)
    assert rel(zp.cpu().numpy(), ref) <= 1e-12


def test_q1_coefficient_hierarchy_levels_match_oracle(cuda, restatement):
    """Rediscretised coarse levels with the reference's Q1 viscosity hierarchy
    (nodal projection, scaled restriction, clamped interpolation,
    src/material_point_utils.c:894-1420): every level operator equals the
    oracle's MatMult with the oracle's restricted viscosity and injected coordinates."""
    from ptatin3d_b200 import COARSE_ETA_Q1
    m, nlev = 8, 3
    c, eta, _ = sinker(m, contrast=1e3, deform=0.1)
    S = StokesSolver(m, m, m, BITS, nlevels=nlev, coarse_op=COARSE_REDISC, coarse_eta=COARSE_ETA_Q1)
    S.setup(c, eta)
    etas = restatement.eta_hierarchy((m, m, m), eta, nlev)
    rng = np.random.default_rng(4)
    cl = c
    for depth in range(nlev):
        mm = m >> depth
        if depth:
            nf = 2 * (2 * mm) + 1
            cl = cl.reshape(nf, nf, nf, 3)[::2, ::2, ::2].reshape(-1).copy()  # injection
        x = rng.uniform(-1, 1, size=3 * (2 * mm + 1) ** 3)
        y = S.level_apply(nlev - 1 - depth, x).cpu().numpy()
        mask = M.dirichlet_mask(mm, mm, mm, BITS)
        ref = matmult_a11(lambda v: restatement.a11_raw((mm, mm, mm), cl, etas[depth], v), x, mask)
        assert rel(y, ref) <= 1e-12, depth


def test_graph_and_eager_preconditioner_agree(cuda):
    m = 8
    c, eta, rho = sinker(m)
    a = StokesSolver(m, m, m, BITS, nlevels=3, use_graph=1)
    b = StokesSolver(m, m, m, BITS, nlevels=3, use_graph=0)
    for s in (a, b):
        s.setup(c, eta)
    rng = np.random.default_rng(0)
    ru = rng.standard_normal(a.nu)
    ru[M.dirichlet_mask(m, m, m, BITS).astype(bool)] = 0.0
    rp = rng.standard_normal(a.np)
    za = a.apply_pc(ru, rp)
    zb = b.apply_pc(ru, rp)
    for x, y in zip(za, zb):
        assert rel(x.cpu().numpy(), y.cpu().numpy()) <= 1e-14


@pytest.mark.parametrize("dims,bits", [((8, 4, 12), M.NO_SLIP), ((12, 8, 4), M.FREE_SLIP_FREE_SURFACE),
                                       ((4, 8, 8), BITS)])
def test_non_cubic_meshes_and_boundary_sets(cuda, restatement, dims, bits):
    """Box meshes with unequal sides and other Dirichlet sets: the converged
    solution satisfies the oracle's assembled system (residual check through the
    oracle operators, no dense assembly needed)."""
    from oracle.oracle import matmult_a12, matmult_a21
    mx, my, mz = dims
    c = M.perturb_interior(M.uniform_coords(mx, my, mz), mx, my, mz, frac=0.1, seed=2)
    qp = M.qp_coords(c, mx, my, mz)
    cen, r = M.random_sinkers(2, 3, 0.2)
    eta, rho = M.sinker_eta(qp, cen, r, 1.0, 10.0), M.sinker_density(qp, cen, r, 1.0, 1.01)
    S = StokesSolver(mx, my, mz, bits, nlevels=3, rtol=1e-10, max_it=600)
    S.setup(c, eta)
    S.set_rhs_body_force(rho)
    u, p, st = S.solve()
    u, p = u.cpu().numpy(), p.cpu().numpy()
    mask = M.dirichlet_mask(mx, my, mz, bits)
    e = eta.reshape(-1)
    ru = matmult_a11(lambda v: restatement.a11_raw(dims, c, e, v), u, mask)
    ru += matmult_a12(lambda v: restatement.a12_raw(dims, c, v), p, mask)
    bu = body_force(restatement, dims, c, rho)
    bu[mask.astype(bool)] = 0.0
    rp = matmult_a21(lambda v: restatement.a21_raw(dims, c, v), u, mask)
    res = np.sqrt(np.linalg.norm(ru - bu) ** 2 + np.linalg.norm(rp) ** 2)
    assert st["converged"] and res <= 1e-9 * np.linalg.norm(bu)


def test_solver_rejects_bad_sizes(cuda):
    with pytest.raises(P3DError):
        StokesSolver(6, 6, 6, BITS, nlevels=3)  # 6 not divisible by 4
    with pytest.raises(P3DError):
        StokesSolver(8, 8, 8, BITS, restart=200)
    with pytest.raises(P3DError):
        StokesSolver(16, 16, 16, BITS, nlevels=1)  # coarse level too large for the dense inverse


def test_setup_waits_for_arrays_written_on_the_callers_stream(cuda, restatement):
    """Coordinates, viscosity and density produced on the caller's (torch's)
    stream just before the calls, with a long queue of unrelated work ahead of
    them: the library reads them on its own stream only after that work, so
    the operators and the right-hand side equal those set up from host arrays."""
    m = 8
    c, eta, rho = sinker(m, deform=0.1)
    busy = torch.rand(1 << 26, dtype=torch.float64, device="cuda")
    for _ in range(40):  # ~0.1 s of queued work on the current stream
        busy.mul_(1.0000001)
    c_d = torch.tensor(c.reshape(-1), device="cuda") * 1.0  # written by kernels behind that queue
    e_d = torch.tensor(eta.reshape(-1), device="cuda") * 1.0
    r_d = torch.tensor(rho.reshape(-1), device="cuda") * 1.0
    S = StokesSolver(m, m, m, BITS, nlevels=2, rtol=1e-9, max_it=200)
    S.setup(c_d, e_d)
    S.set_rhs_body_force(r_d)
    u_d, p_d, _ = S.solve()
    H = StokesSolver(m, m, m, BITS, nlevels=2, rtol=1e-9, max_it=200)
    H.setup(c, eta)
    H.set_rhs_body_force(rho)
    u_h, p_h, _ = H.solve()
    x = np.random.default_rng(0).uniform(-1, 1, size=c.size)
    yd, yh = S.level_apply(1, x), H.level_apply(1, x)
    assert rel(yd.cpu().numpy(), yh.cpu().numpy()) <= 1e-14  # brick-face atomics: rounding-order differences only
    # both solves stop at rtol 1e-9 on the same system; their iterates differ by
    # the summation order of the atomics, amplified by the conditioning
    assert rel(u_d.cpu().numpy(), u_h.cpu().numpy()) <= 1e-5
    assert rel(p_d.cpu().numpy(), p_h.cpu().numpy()) <= 1e-5
    S.destroy()
    H.destroy()


@pytest.mark.parametrize("prec", [PREC_F64, PREC_F32])
def test_inner_tolerance_loop_graph_and_eager_agree(cuda, prec):
    """The tolerance-driven inner velocity solve runs as a conditional WHILE
    node inside the captured preconditioner graph, and as a host loop without
    the graph: the same outer and inner iteration counts (up to the rounding
    order of atomics) and the same solution."""
    m = 16
    c, eta, rho = sinker(m, nsph=4, radius=0.15, contrast=1e2)
    out = {}
    for graph in (1, 0):
        S = StokesSolver(m, m, m, BITS, nlevels=3, rtol=1e-8, max_it=300, mg_precision=prec, inner_rtol=1e-2,
                         inner_its=60, use_graph=graph, schur_eta=SCHUR_ETA_GEOMEAN)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        u, p, st = S.solve()
        out[graph] = (u.cpu().numpy(), p.cpu().numpy(), st)
        S.destroy()
    (ug, pg, sg), (ue, pe, se) = out[1], out[0]
    assert sg["converged"] and se["converged"]
    # the atomics' summation order changes from run to run, and the FP32
    # multigrid carries it into the Krylov path: counts agree to 10 %
    assert abs(sg["iterations"] - se["iterations"]) <= 0.1 * se["iterations"] + 2
    assert abs(sg["inner_iterations"] - se["inner_iterations"]) <= 0.1 * se["inner_iterations"] + 3
    assert sg["iterations"] < sg["inner_iterations"] <= 60 * sg["iterations"]
    assert rel(ug, ue) <= 1e-6 and rel(pg, pe) <= 1e-6


def test_inner_tolerance_cap_ends_the_loop(cuda):
    """An unreachable inner tolerance stops at inner_its iterations per
    preconditioner application (the device loop's bound), and the outer
    iteration still converges."""
    m = 8
    c, eta, rho = sinker(m, contrast=1e2)
    S = StokesSolver(m, m, m, BITS, nlevels=2, rtol=1e-8, max_it=100, inner_rtol=1e-300, inner_its=3)
    S.setup(c, eta)
    S.set_rhs_body_force(rho)
    _, _, st = S.solve()
    assert st["converged"]
    assert st["inner_iterations"] == 3 * st["iterations"]  # one preconditioner application per outer iteration


@pytest.mark.parametrize("prec", [PREC_F64, PREC_F32])
def test_grouped_solve_equals_member_solves(cuda, prec):
    """Four solvers of one mesh shape with different sinkers solved together
    (one launch per kernel for all four, lock-step FGMRES): each member takes
    its own solve's iteration count and reaches its solution; a member whose
    density holds a NaN breaks down alone, and an easy member leaves the group
    early while the others go on."""
    from ptatin3d_b200 import _lib
    from ptatin3d_b200.solver import solve_grouped
    m = 16
    cases = [sinker(m, nsph=2, radius=0.15, contrast=1e2, seed=s) for s in (1, 2, 3)]
    cases.append(sinker(m, nsph=1, radius=0.1, contrast=2.0, seed=4))  # converges much sooner
    kw = dict(nlevels=3, rtol=1e-9, max_it=600, mg_precision=prec, schur_eta=SCHUR_ETA_GEOMEAN)
    alone = []
    for c, eta, rho in cases:
        S = StokesSolver(m, m, m, BITS, **kw)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        u, p, st = S.solve()
        alone.append((u.cpu().numpy(), p.cpu().numpy(), st))
        S.destroy()
    group = []
    for c, eta, rho in cases:
        S = StokesSolver(m, m, m, BITS, **kw)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        group.append(S)
    c, eta, rho = cases[0]
    bad = StokesSolver(m, m, m, BITS, **kw)
    bad.setup(c, eta)
    rho_nan = rho.copy()
    rho_nan[40, 5] = np.nan
    bad.set_rhs_body_force(rho_nan)
    res = solve_grouped(group + [bad])
    for (u, p, st, status), (ua, pa, sa) in zip(res[:4], alone):
        assert status == 0 and st["converged"]
        assert abs(st["iterations"] - sa["iterations"]) <= max(2, 0.05 * sa["iterations"])
        assert rel(u.cpu().numpy(), ua) <= 1e-6 and rel(p.cpu().numpy(), pa) <= 1e-5
    assert res[3][2]["iterations"] < res[0][2]["iterations"]
    assert res[4][3] == _lib.P3D_ERR_BREAKDOWN
    for S in group + [bad]:
        S.destroy()
