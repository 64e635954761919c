"""Results do not depend on the former contents of reused device memory.

With p3d_debug_poison_allocations(fill) every device allocation of the
library starts filled with one byte value: 0xFF (every double a NaN) or 0x40
(every double 32.5, every float 3.0).  A kernel that reads a buffer before
writing it then gives NaNs or a different iteration count instead of
depending on what an earlier object left behind.  NaNs alone do not find
everything: a stale |w|^2 in the Gram-Schmidt step is only used when it
passes a comparison, which a NaN (or a zero from fresh memory) never does
but 32.5 does.  Each case is solved from fresh allocations and from
poisoned ones and must give the same iterations and solution.
"""
import json
import os

import numpy as np
import pytest
import torch

from cases import bump_case, rel, sinker_markers
from ptatin3d_b200 import (COARSE_ETA_Q1, COARSE_GALERKIN, COARSE_REDISC, PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN,
                           SCHUR_ETA_QP, _lib)
from ptatin3d_b200 import mesh as M
from ptatin3d_b200.solver import StokesSolver, solve_grouped

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
APP = json.load(open(os.path.join(HERE, "golden", "application_expected.json")))
BITS = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)


FILLS = [0xFF, 0x40]
OFF = -1


@pytest.fixture
def poison():
    L = _lib.lib()
    yield lambda fill: L.p3d_debug_poison_allocations(fill)
    L.p3d_debug_poison_allocations(OFF)


def sinker(m, seed, contrast=1e2):
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(2, seed, 0.15)
    return c, M.sinker_eta(qp, cen, r, 1.0, contrast), M.sinker_density(qp, cen, r, 1.0, 1.01)


def _solve(m, case, nodal=None, **kw):
    c, eta, rho = case
    S = StokesSolver(m, m, m, BITS, **kw)
    S.setup(c, eta, eta_nodes=nodal)
    S.set_rhs_body_force(rho)
    u, p, st = S.solve(raise_on_noconv=False)
    S.destroy()
    return u.cpu().numpy(), p.cpu().numpy(), st


def _same(a, b, mixed=False):
    """Same solve: FP64 preconditioners repeat to rounding (the brick-face
    atomics add in varying order); FP32 ones amplify that order into a few
    iterations more or less at rtol 1e-8."""
    (ua, pa, sa), (ub, pb, sb) = a, b
    assert np.isfinite(ub).all() and np.isfinite(pb).all()
    assert sb["converged"] == sa["converged"]
    dits = max(2, 0.1 * sa["iterations"]) if mixed else 2
    assert abs(sb["iterations"] - sa["iterations"]) <= dits, (sa["iterations"], sb["iterations"])
    tu, tp = (3e-5, 1e-4) if mixed else (1e-6, 1e-5)
    assert rel(ub, ua) <= tu and rel(pb, pa) <= tp


OPTION_SETS = {
    "galerkin_inner_rtol_graph": dict(nlevels=3, cheb_its=10, rtol=1e-3, max_it=100, inner_rtol=1e-2, inner_its=200,
                                      coarse_op=COARSE_GALERKIN, schur_eta=SCHUR_ETA_QP),
    "galerkin_inner_rtol_eager": dict(nlevels=3, cheb_its=10, rtol=1e-3, max_it=100, inner_rtol=1e-2, inner_its=200,
                                      coarse_op=COARSE_GALERKIN, schur_eta=SCHUR_ETA_QP, use_graph=0),
    "mixed_redisc_inner_cg2": dict(nlevels=3, rtol=1e-8, max_it=300, mg_precision=PREC_F32, coarse_op=COARSE_REDISC,
                                   inner_its=2, schur_eta=SCHUR_ETA_GEOMEAN),
    "one_level": dict(nlevels=1, rtol=1e-8, max_it=300),
    "fp64_default": dict(nlevels=3, rtol=1e-8, max_it=300, mg_precision=PREC_F64),
}


@pytest.mark.parametrize("fill", FILLS)
@pytest.mark.parametrize("name", sorted(OPTION_SETS))
def test_solves_from_poisoned_allocations_equal_fresh_ones(cuda, poison, name, fill):
    m = 8
    case = sinker(m, seed=3)
    kw = OPTION_SETS[name]
    poison(OFF)
    fresh = _solve(m, case, **kw)
    poison(fill)
    _same(fresh, _solve(m, case, **kw), mixed=kw.get("mg_precision") == PREC_F32)


@pytest.mark.parametrize("fill", FILLS)
def test_application_solve_from_poisoned_allocations(cuda, poison, fill):
    """The viscous-sinker application solve (device marker projection, the
    reference's solver options) takes the same outer iterations whatever the
    reused memory held."""
    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    rec = APP["sinker_galerkin_8x8x8"]
    case = bump_case(rec["mx"], rec["my"], rec["mz"])
    wil, xi, eta_p, rho_p = sinker_markers(case, rec["eta0"], rec["eta1"], rec["rho0"], rec["rho1"])
    d = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)
    res = []
    for f in (OFF, fill):
        poison(f)
        eta_q, rho_q = update_gauss_properties(case["dims"], PROJ_Q1, d(wil, torch.int32), d(xi, torch.float64),
                                               d(eta_p, torch.float64), d(rho_p, torch.float64))
        S = StokesSolver(*case["dims"], case["bits"], nlevels=rec["nlevels"], cheb_its=rec["cheb_its"],
                         rtol=rec["ksp_rtol"], max_it=100, inner_rtol=rec["inner_rtol"], inner_its=200,
                         schur_eta=SCHUR_ETA_QP)
        S.setup(d(case["coords"], torch.float64), eta_q)
        S.set_rhs_body_force(rho_q, (0.0, 1.0, 0.0))
        u, p, st = S.solve()
        S.destroy()
        res.append((u.cpu().numpy(), p.cpu().numpy(), st))
    _same(*res)
    assert abs(res[1][2]["iterations"] - rec["outer_iterations"]) <= 3


@pytest.mark.parametrize("fill", FILLS)
def test_nodal_hierarchy_from_poisoned_allocations(cuda, poison, fill):
    m = 8
    c, eta, rho = sinker(m, seed=5)
    v = np.ones((2 * m + 1) ** 3) * 3.0
    kw = dict(nlevels=3, rtol=1e-8, max_it=300, coarse_op=COARSE_REDISC, coarse_eta=COARSE_ETA_Q1)
    poison(OFF)
    fresh = _solve(m, (c, eta, rho), nodal=v, **kw)
    poison(fill)
    _same(fresh, _solve(m, (c, eta, rho), nodal=v, **kw))


@pytest.mark.parametrize("fill", FILLS)
@pytest.mark.parametrize("prec", [PREC_F64, PREC_F32])
def test_grouped_solve_from_poisoned_allocations(cuda, poison, prec, fill):
    m = 8
    cases = [sinker(m, seed=s) for s in (1, 2, 3)]
    kw = dict(nlevels=3, rtol=1e-8, max_it=300, mg_precision=prec, schur_eta=SCHUR_ETA_GEOMEAN)
    out = []
    for f in (OFF, fill):
        poison(f)
        group = []
        for c, eta, rho in cases:
            S = StokesSolver(m, m, m, BITS, **kw)
            S.setup(c, eta)
            S.set_rhs_body_force(rho)
            group.append(S)
        res = solve_grouped(group)
        out.append([(u.cpu().numpy(), p.cpu().numpy(), st) for u, p, st, _ in res])
        for S in group:
            S.destroy()
    for a, b in zip(*out):
        _same(a, b, mixed=prec == PREC_F32)


@pytest.mark.parametrize("fill", FILLS)
def test_operator_apply_from_poisoned_allocations(cuda, poison, fill):
    from ptatin3d_b200.operators import MatStokesMF, mesh_desc_whole
    m = 8
    c, eta, _ = sinker(m, seed=2)
    c = M.perturb_interior(c, m, m, m, frac=0.1, seed=2)
    rng = np.random.default_rng(0)
    nu = 3 * (2 * m + 1) ** 3
    x = torch.tensor(rng.standard_normal(nu), device=cuda)
    out = []
    for f in (OFF, fill):
        poison(f)
        op = MatStokesMF(mesh_desc_whole(m, m, m, BITS))
        op.set_coefficients(torch.tensor(c, device=cuda), torch.tensor(eta, device=cuda))
        y = torch.empty_like(x)
        op.mult(x, y)
        d = torch.empty_like(x)
        op.get_diagonal(d)
        out.append((y.cpu().numpy(), d.cpu().numpy()))
        op.destroy()
    assert np.isfinite(out[1][0]).all() and np.isfinite(out[1][1]).all()
    assert rel(out[1][0], out[0][0]) <= 1e-13 and rel(out[1][1], out[0][1]) <= 1e-14


@pytest.mark.parametrize("fill", FILLS)
def test_served_requests_from_poisoned_allocations(cuda, poison, fill):
    """Requests solved by the server (pool slots, grouped solves of
    same-shape requests) give the same results on poisoned allocations."""
    from ptatin3d_b200.serving import StokesServer
    from test_gpu_serving import request, submit
    reqs = [(8, request(8, 2, 1e2, s)) for s in (1, 2, 3)] + [(12, request(12, 2, 1e2, 4))]
    out = []
    for f in (OFF, fill):
        poison(f)
        with StokesServer(hbm_budget=4 << 30, max_active=4) as S:
            for t, (m, arr) in enumerate(reqs):
                submit(S, m, arr, t, rtol=1e-10)
            out.append({r["tag"]: r for r in S.wait_all()})
    for t in range(len(reqs)):
        a, b = out[0][t], out[1][t]
        assert a["ok"] and b["ok"], (a, b)
        assert abs(a["iterations"] - b["iterations"]) <= 2
        assert rel(b["u"], a["u"]) <= 1e-6 and rel(b["p"], a["p"]) <= 1e-5
