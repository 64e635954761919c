"""GPU parity of the sm_100a operators against the CPU oracle.

Tolerances (FP64): 1e-12 relative in the 2-norm, the bar named for the A11
apply; FP32 operators: 1e-5 relative against the FP64 result.
"""
import json
import math
import os

import numpy as np
import pytest
import torch

from cases import bump_case, rel, sinker_case
from oracle.oracle import get_diagonal, matmult_a11, matmult_a12, matmult_a21
from ptatin3d_b200 import GEOM_AFFINE, GEOM_GENERAL, PREC_F32, PREC_F64
from ptatin3d_b200 import mesh as M
from ptatin3d_b200.operators import MatStokesMF, mesh_desc_whole, mg_prolong, mg_restrict

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 1e-5


def make_op(case, prec=PREC_F64, geom=0):
    d = mesh_desc_whole(*case["dims"], case["bits"])
    op = MatStokesMF(d, prec)
    op.set_coefficients(case["coords"], case["eta"], geom)
    return op


def T(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.double().cpu().numpy()


@pytest.mark.parametrize("dims", [(8, 9, 11), (1, 1, 1), (1, 1, 3), (7, 3, 5), (6, 4, 9)])
@pytest.mark.parametrize("geom", [GEOM_GENERAL, GEOM_AFFINE])
def test_a11_raw_matches_oracle(cuda, restatement, dims, geom):
    case = bump_case(*dims, eta_kind="random", seed=sum(dims))
    if geom == GEOM_AFFINE:  # affine mesh for the affine path
        case["coords"] = M.uniform_coords(*dims, hi=(1.0, 2.0, 0.5))
    op = make_op(case, geom=geom)
    assert op.geometry_mode == geom
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, size=case["coords"].size)
    y = torch.zeros(x.size, dtype=torch.float64, device="cuda")
    op.spmv(T(x), y)
    ref = restatement.a11_raw(case["dims"], case["coords"], case["eta"].reshape(-1), x)
    assert rel(host(y), ref) <= TOL64


def test_a11_auto_detects_affine(cuda):
    case = sinker_case(10)
    assert make_op(case).geometry_mode == GEOM_AFFINE
    case = sinker_case(10, deform=0.2)
    assert make_op(case).geometry_mode == GEOM_GENERAL


@pytest.mark.parametrize("deform", [0.0, 0.2])
def test_a11_matmult_sinker(cuda, restatement, deform):
    case = sinker_case(12, deform=deform)
    op = make_op(case)
    y = torch.full((case["x"].size,), float("nan"), dtype=torch.float64, device="cuda")  # overwritten, never read
    op.mult(T(case["x"]), y)
    d, c, e = case["dims"], case["coords"], case["eta"].reshape(-1)
    ref = matmult_a11(lambda v: restatement.a11_raw(d, c, e, v), case["x"], case["mask"])
    assert rel(host(y), ref) <= TOL64


def test_affine_and_general_paths_agree(cuda):
    case = sinker_case(11)
    yA = torch.empty(case["x"].size, dtype=torch.float64, device="cuda")
    yG = torch.empty_like(yA)
    make_op(case, geom=GEOM_AFFINE).mult(T(case["x"]), yA)
    make_op(case, geom=GEOM_GENERAL).mult(T(case["x"]), yG)
    assert rel(host(yA), host(yG)) <= 1e-13


GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_expected.json")))


@pytest.mark.parametrize("name", ["compare_mf_asm_8x9x11", "avx_cuda/compare_mf_1x1x3_p3",
                                  "avx_cuda/compare_mf_16x16x16_p24", "compare_mf_asm_17x11x13_p27"])
def test_reference_expected_on_gpu(cuda, name):
    """The reference's printed y.y values, reproduced by the GPU operators."""
    rec = GOLD[name]
    dims = (rec["mx"], rec["my"], rec["mz"])
    case = bump_case(*dims)
    op = make_op(case)
    nv, npr = op.n_velocity, op.n_pressure
    x, p = T(case["x"]), T(case["p"])
    y = torch.empty(nv, dtype=torch.float64, device="cuda")
    yp = torch.empty(npr, dtype=torch.float64, device="cuda")
    d = torch.empty(nv, dtype=torch.float64, device="cuda")
    checks = {}
    op.mult_a21(x, yp)
    checks["A21"] = host(yp)
    op.mult_a12(p, y)
    checks["A12"] = host(y)
    if rec["eta1"] == 1.0 or dims == (1, 1, 3):
        op.mult(x, y)
        checks["A11"] = host(y)
        op.get_diagonal(d)
        checks["diagA11"] = host(d)
    for k, v in checks.items():
        gold = float(rec[k])
        val = float(v @ v)
        if math.isnan(gold):
            assert math.isnan(val)
        else:
            assert abs(val - gold) <= 5e-9 * abs(gold), (k, val, gold)


SHEAR = np.array([[1.0, 0.3, 0.1], [0.2, 1.2, -0.15], [0.05, 0.25, 0.9]])


@pytest.mark.parametrize("deform,shear", [(0.0, False), (0.0, True), (0.15, False)])
def test_diagonal_a12_a21_fused(cuda, restatement, deform, shear):
    """diag(A11), A12, A21 and the fused operator against the oracle: on the
    uniform and the sheared (affine, off-diagonal Jacobian) mesh through the
    per-element-Jacobian kernels, on the perturbed mesh through the general ones."""
    case = sinker_case(6, deform=deform, seed=4)
    if shear:
        case["coords"] = (case["coords"].reshape(-1, 3) @ SHEAR.T + 0.5).reshape(-1)
    d, c, e, mask = case["dims"], case["coords"], case["eta"].reshape(-1), case["mask"]
    op = make_op(case)
    assert op.geometry_mode == (GEOM_GENERAL if deform else GEOM_AFFINE)
    nv, npr = op.n_velocity, op.n_pressure
    x, p = T(case["x"]), T(case["p"])
    dg = torch.empty(nv, dtype=torch.float64, device="cuda")
    op.get_diagonal(dg)
    assert rel(host(dg), get_diagonal(lambda: restatement.diag_raw(d, c, e), mask)) <= TOL64
    yu = torch.empty(nv, dtype=torch.float64, device="cuda")
    op.mult_a12(p, yu)
    assert rel(host(yu), matmult_a12(lambda v: restatement.a12_raw(d, c, v), case["p"], mask)) <= TOL64
    yp = torch.empty(npr, dtype=torch.float64, device="cuda")
    op.mult_a21(x, yp)
    assert rel(host(yp), matmult_a21(lambda v: restatement.a21_raw(d, c, v), case["x"], mask)) <= TOL64
    # fused [A11 A12; A21 0]
    fu, fp = torch.empty_like(yu), torch.empty_like(yp)
    op.mult_stokes(x, p, fu, fp)
    ref_u = matmult_a11(lambda v: restatement.a11_raw(d, c, e, v), case["x"], mask)
    ref_u += matmult_a12(lambda v: restatement.a12_raw(d, c, v), case["p"], mask)
    ref_u[mask.astype(bool)] = case["x"][mask.astype(bool)]
    assert rel(host(fu), ref_u) <= TOL64
    assert rel(host(fp), host(yp)) <= TOL64


def test_low_order_operator_matches_reference_golden(cuda):
    """MatMult_MFStokes_A11LowOrder (ONEPOINTQ: the Jacobian of the element centre
    at every Gauss point, src/stokes_operators_mf.c:353-488): the affine path
    forced on a deformed mesh, against the reference's own kernel output."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "loworder_4x3x5.npz"))
    dims = tuple(int(v) for v in g["dims"])
    case = dict(dims=dims, coords=g["coords"], eta=g["eta"], bits=M.FREE_SLIP)
    op = make_op(case, geom=GEOM_AFFINE)
    y = torch.zeros(g["x"].size, dtype=torch.float64, device="cuda")
    op.spmv(T(g["x"]), y)
    assert rel(host(y), g["y"]) <= TOL64


def test_low_order_operator_matches_reference_kernel(cuda, reference_kernels):
    m = 6
    c = M.perturb_interior(M.uniform_coords(m, m, m), m, m, m, frac=0.2, seed=1)
    eta = 10 ** np.random.default_rng(2).uniform(-1, 1, size=(m ** 3, 27))
    reference_kernels.setup((m, m, m), c, eta)
    x = np.random.default_rng(3).uniform(-1, 1, size=c.size)
    op = make_op(dict(dims=(m, m, m), coords=c, eta=eta, bits=M.FREE_SLIP), geom=GEOM_AFFINE)
    y = torch.zeros(x.size, dtype=torch.float64, device="cuda")
    op.spmv(T(x), y)
    assert rel(host(y), reference_kernels.a11_raw(x, "loworder")) <= TOL64


@pytest.mark.parametrize("deform,with_forces", [(0.15, True), (0.0, True), (0.15, False)])
def test_stokes_residual_matches_oracle(cuda, restatement, deform, with_forces):
    """FormFunction_Stokes (src/stokes_form_function.c:99-564) on the GPU against
    the oracle: Dirichlet values inserted, body forces from Gauss-point Fu / Fp,
    Dirichlet rows u_k - phi_k."""
    from oracle.oracle import stokes_residual
    case = sinker_case(6, deform=deform, seed=4)
    d, c, e, mask = case["dims"], case["coords"], case["eta"], case["mask"]
    op = make_op(case)
    rng = np.random.default_rng(9)
    nel = d[0] * d[1] * d[2]
    u, p = case["x"], case["p"]
    phi = rng.uniform(-1, 1, size=u.size)
    fu = rng.uniform(-1, 1, size=(nel, 27, 3)) if with_forces else None
    fp = rng.uniform(-1, 1, size=(nel, 27)) if with_forces else None
    ru, rp = op.residual(u, p, fu=fu, fp=fp, phi=phi if with_forces else None)
    zero_u, zero_p = np.zeros((nel, 27, 3)), np.zeros((nel, 27))
    ref_u, ref_p = stokes_residual(restatement, d, c, e, mask, u, p, phi if with_forces else np.zeros(u.size),
                                   fu if with_forces else zero_u, fp if with_forces else zero_p)
    assert rel(host(ru), ref_u) <= TOL64
    assert rel(host(rp), ref_p) <= TOL64


@pytest.mark.parametrize("deform", [0.0, 0.2])
def test_fp32_operator(cuda, deform):
    case = sinker_case(16, deform=deform, eta1=1e2)
    y64 = torch.empty(case["x"].size, dtype=torch.float64, device="cuda")
    make_op(case).mult(T(case["x"]), y64)
    op32 = make_op(case, prec=PREC_F32)
    y32 = torch.empty(case["x"].size, dtype=torch.float32, device="cuda")
    op32.mult(T(case["x"], torch.float32), y32)
    assert rel(host(y32), host(y64)) <= TOL32


@pytest.mark.parametrize("deform", [0.0, 0.2])
def test_fp32_pressure_coupling(cuda, deform):
    """FP32 A12, A21 and the fused operator against FP64 (affine and general kernels)."""
    case = sinker_case(12, deform=deform, eta1=1e2)
    op64, op32 = make_op(case), make_op(case, prec=PREC_F32)
    x64, p64 = T(case["x"]), T(case["p"])
    x32, p32 = T(case["x"], torch.float32), T(case["p"], torch.float32)
    nv, npr = op64.n_velocity, op64.n_pressure
    out = {}
    for name, op, x, p, dt in (("64", op64, x64, p64, torch.float64), ("32", op32, x32, p32, torch.float32)):
        yu = torch.empty(nv, dtype=dt, device="cuda")
        yp = torch.empty(npr, dtype=dt, device="cuda")
        op.mult_a12(p, yu)
        op.mult_a21(x, yp)
        fu, fp = torch.empty_like(yu), torch.empty_like(yp)
        op.mult_stokes(x, p, fu, fp)
        out[name] = [host(v) for v in (yu, yp, fu, fp)]
    for a, b in zip(out["32"], out["64"]):
        assert rel(a, b) <= TOL32


def test_host_apply_matches_device(cuda):
    case = sinker_case(9, deform=0.1)
    op = make_op(case)
    yd = torch.zeros(case["x"].size, dtype=torch.float64, device="cuda")
    op.spmv(T(case["x"]), yd)
    yh = np.full(case["x"].size, 7.0)  # overwritten, as the reference backend's copy-out does
    op.mult_host(case["x"], yh)
    assert rel(yh, host(yd)) <= 1e-15


@pytest.mark.parametrize("dims,deform,chunks", [((7, 3, 11), 0.2, 5), ((7, 3, 11), 0.0, 5), ((5, 6, 8), 0.1, 16),
                                                ((6, 5, 4), 0.0, 2)])
def test_host_apply_chunked_pipeline(cuda, restatement, dims, deform, chunks):
    """The z-chunked host apply (copies overlapped with the applies) equals the
    oracle MatMult for any chunk count, brick height (affine 4, general 2) and
    ragged last chunk."""
    from ptatin3d_b200 import _lib
    mx, my, mz = dims
    c = M.uniform_coords(mx, my, mz)
    if deform:
        c = M.perturb_interior(c, mx, my, mz, frac=deform, seed=3)
    rng = np.random.default_rng(7)
    eta = 10.0 ** rng.uniform(-1, 1, size=(mx * my * mz, 27))
    case = dict(dims=dims, coords=c, eta=eta, bits=M.FREE_SLIP)
    op = make_op(case)
    assert op.geometry_mode == (GEOM_GENERAL if deform else GEOM_AFFINE)
    _lib.check(_lib.lib().p3d_op_set_host_chunks(op.h, chunks))
    x = rng.uniform(-1, 1, size=c.size)
    y = np.full(c.size, np.nan)
    op.mult_host(x, y, boundary=True)
    ref = matmult_a11(lambda v: restatement.a11_raw(dims, c, eta.reshape(-1), v), x, M.dirichlet_mask(*dims, M.FREE_SLIP))
    assert rel(y, ref) <= TOL64


def test_host_apply_registered_pageable(cuda, restatement):
    """p3d_a11_apply_host on pageable arrays, with the operator page-locking
    them on first use: the same result as without, on repeated calls, and the
    arrays are released again when registration is switched off."""
    from ptatin3d_b200 import _lib
    case = sinker_case(10, deform=0.2)
    op = make_op(case)
    _lib.check(_lib.lib().p3d_op_set_bc_mode(op.h, _lib.BC_MATMULT))
    x = np.ascontiguousarray(case["x"])
    y0 = np.full(x.size, np.nan)
    op.mult_host(x, y0, boundary=True)
    y = np.empty(x.size)  # registered arrays stay allocated until registration is switched off
    _lib.check(_lib.lib().p3d_op_set_host_register(op.h, 1))
    for _ in range(3):
        y[:] = np.nan
        op.mult_host(x, y, boundary=True)
        assert not np.isnan(y).any()
        assert rel(y, y0) <= 1e-15
    _lib.check(_lib.lib().p3d_op_set_host_register(op.h, 0))
    d, c, e = case["dims"], case["coords"], case["eta"].reshape(-1)
    assert rel(y0, matmult_a11(lambda v: restatement.a11_raw(d, c, e, v), x, case["mask"])) <= TOL64


def test_operator_properties_large(cuda):
    """Size-independent properties at 64^3 (6.4M dofs): symmetry and linearity."""
    m = 64
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    eta = M.layered_eta(qp, seed=3)
    case = dict(dims=(m, m, m), coords=c, eta=eta, bits=M.FREE_SLIP)
    op = make_op(case)
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.rand(op.n_velocity, dtype=torch.float64, device="cuda", generator=g) - 0.5
    b = torch.rand(op.n_velocity, dtype=torch.float64, device="cuda", generator=g) - 0.5
    Aa, Ab, Ac = torch.empty_like(a), torch.empty_like(a), torch.empty_like(a)
    op.mult(a, Aa)
    op.mult(b, Ab)
    op.mult(2.0 * a - 3.0 * b, Ac)
    assert abs(float(b @ Aa - a @ Ab)) <= 1e-11 * float(a.norm() * Aa.norm())
    assert float((Ac - (2.0 * Aa - 3.0 * Ab)).norm()) <= 1e-13 * float(Ac.norm())
    Aa2 = torch.empty_like(a)
    op.mult(a, Aa2)
    assert float((Aa2 - Aa).norm()) <= 1e-15 * float(Aa.norm())  # run-to-run (face atomics) agreement


def test_mg_transfer(cuda, restatement):
    rng = np.random.default_rng(0)
    cn = (5, 4, 6)
    fn = [2 * c - 1 for c in cn]
    xc = rng.standard_normal(3 * int(np.prod(cn)))
    xf = rng.standard_normal(3 * int(np.prod(fn)))
    for dt, tol in ((torch.float64, 1e-15), (torch.float32, 1e-6)):
        gf = torch.empty(xf.size, dtype=dt, device="cuda")
        mg_prolong(T(xc, dt), gf, cn)
        assert rel(host(gf), restatement.prolong(cn, 3, xc)) <= tol
        gc = torch.empty(xc.size, dtype=dt, device="cuda")
        mg_restrict(T(xf, dt), gc, cn)
        assert rel(host(gc), restatement.restrict(cn, 3, xf)) <= tol


@pytest.mark.parametrize("deform", [0.0, 0.15])
def test_ghosted_local_arrays(cuda, restatement, deform):
    """The drop-in layout: a rank's elements inside a ghosted node lattice
    (PETSc local vectors, ghost layers of 2 nodes on some sides, faces of the
    local block not on the global boundary).  The raw element apply, A12 and
    A21 must equal the oracle on the owned sub-lattice and leave every
    ghost-only entry untouched."""
    mx, my, mz = 4, 3, 5
    lo, hi = (2, 0, 2), (2, 2, 0)  # ghost nodes before / after the owned block
    gx, gy, gz = (2 * m + 1 + a + b for m, a, b in zip((mx, my, mz), lo, hi))
    full = M.uniform_coords(gx // 2, gy // 2, gz // 2)  # any lattice of the right extent works for ghosts
    c = full.reshape(gz, gy, gx, 3).copy()
    owned = (slice(lo[2], lo[2] + 2 * mz + 1), slice(lo[1], lo[1] + 2 * my + 1), slice(lo[0], lo[0] + 2 * mx + 1))
    c_loc = M.uniform_coords(mx, my, mz)
    if deform:
        c_loc = M.perturb_interior(c_loc, mx, my, mz, frac=deform, seed=3)
    c[owned] = c_loc.reshape(2 * mz + 1, 2 * my + 1, 2 * mx + 1, 3)
    rng = np.random.default_rng(5)
    eta = 10 ** rng.uniform(-1, 1, size=(mx * my * mz, 27))
    x = rng.uniform(-1, 1, size=(gz, gy, gx, 3))
    p = rng.uniform(-1, 1, size=4 * mx * my * mz)
    d = mesh_desc_whole(mx, my, mz, M.FREE_SLIP)
    d.gx, d.gy, d.gz = gx, gy, gz
    d.ox, d.oy, d.oz = lo
    d.global_faces = 0  # an interior rank: no Dirichlet face
    op = MatStokesMF(d, PREC_F64)
    op.set_coefficients(c.reshape(-1), eta)
    assert op.geometry_mode == (GEOM_GENERAL if deform else GEOM_AFFINE)
    y = torch.zeros(x.size, dtype=torch.float64, device="cuda")
    op.spmv(T(x.reshape(-1)), y)
    dims = (mx, my, mz)
    xl = x[owned].reshape(-1)
    ref = restatement.a11_raw(dims, c_loc, eta.reshape(-1), xl)
    yh = host(y).reshape(gz, gy, gx, 3)
    assert rel(yh[owned].reshape(-1), ref) <= TOL64
    ghost = np.ones((gz, gy, gx), dtype=bool)
    ghost[owned] = False
    assert np.all(yh[ghost] == 0.0)
    yu = torch.zeros(x.size, dtype=torch.float64, device="cuda")
    op.mult_a12(T(p), yu, boundary=False)
    yuh = host(yu).reshape(gz, gy, gx, 3)
    assert rel(yuh[owned].reshape(-1), restatement.a12_raw(dims, c_loc, p)) <= TOL64
    assert np.all(yuh[ghost] == 0.0)
    yp = torch.zeros(p.size, dtype=torch.float64, device="cuda")
    op.mult_a21(T(x.reshape(-1)), yp, boundary=False)
    assert rel(host(yp), restatement.a21_raw(dims, c_loc, xl)) <= TOL64


def test_full_size_deformed_apply_matches_reference_kernel(cuda, reference_kernels):
    """The benchmark workload at full size (96^3 deformed mesh, 21.6M dofs,
    log-normal eta over 12 decades): the GPU apply against the reference's own
    MFStokesWrapper_A11_AVX on the same inputs, and symmetry/linearity."""
    m = 96
    c = M.perturb_interior(M.uniform_coords(m, m, m), m, m, m, frac=0.2, seed=4)
    eta = M.lognormal_grf_eta(m, m, m, seed=4, sigma_decades=2.0, corr_len=0.1)
    x = np.random.default_rng(4).uniform(-1.0, 1.0, size=c.size)
    op = make_op(dict(dims=(m, m, m), coords=c, eta=eta, bits=M.FREE_SLIP))
    assert op.geometry_mode == GEOM_GENERAL
    y = torch.zeros(x.size, dtype=torch.float64, device="cuda")
    op.spmv(T(x), y)
    reference_kernels.setup((m, m, m), c, eta)
    assert rel(host(y), reference_kernels.a11_raw(x, "avx")) <= TOL64
    g = torch.Generator(device="cuda").manual_seed(1)
    a = torch.rand(x.size, dtype=torch.float64, device="cuda", generator=g) - 0.5
    Aa, Ax = torch.empty_like(a), torch.empty_like(a)
    op.mult(a, Aa)
    xd = T(x)
    op.mult(xd, Ax)
    assert abs(float(xd @ Aa - a @ Ax)) <= 1e-11 * float(a.norm() * Ax.norm())


def test_c1_sinker_apply_matches_reference_kernel(cuda, reference_kernels):
    """The plain-apply configuration exactly: a 16^3 mesh of affine hexahedra
    (107,811 dofs), eta 1 with 1e3 inside 8 spheres of radius 0.1 whose centres
    are uniform from the seed, x uniform in [-1, 1] from the same seed, free
    slip on all six faces; the GPU MatMult (Dirichlet columns zeroed, rows
    y_k = x_k) against MatMult_MFStokes_A11 over the reference's own
    MFStokesWrapper_A11_AVX (src/stokes_operators.c:1142-1205,
    src/stokes_operators_avx.c:206-315) on the same inputs."""
    case = sinker_case(16, seed=1, nsph=8, radius=0.1, eta1=1e3)
    assert case["x"].size == 107811
    op = make_op(case)
    assert op.geometry_mode == GEOM_AFFINE
    y = torch.full((case["x"].size,), float("nan"), dtype=torch.float64, device="cuda")
    op.mult(T(case["x"]), y)
    reference_kernels.setup(case["dims"], case["coords"], case["eta"])
    ref = matmult_a11(lambda v: reference_kernels.a11_raw(v, "avx"), case["x"], case["mask"])
    assert rel(host(y), ref) <= TOL64
    # the raw element apply (SpMVOp contract, y += A x) as well
    y0 = np.random.default_rng(2).uniform(-1, 1, size=case["x"].size)
    z = T(y0)
    op.spmv(T(case["x"]), z)
    assert rel(host(z), y0 + reference_kernels.a11_raw(case["x"], "avx")) <= TOL64


def test_c3_layered_apply_matches_reference_kernel(cuda, reference_kernels):
    """The layered 64^3 configuration (6.4M dofs; log10 eta uniform in [-3, 3]
    per each of 6 horizontal layers plus 16 inclusions) on the affine path, in
    FP64 against the reference's MFStokesWrapper_A11_AVX, and the FP32
    operator against the FP64 one."""
    m = 64
    c = M.uniform_coords(m, m, m)
    eta = M.layered_eta(M.qp_coords(c, m, m, m), seed=4)
    case = dict(dims=(m, m, m), coords=c, eta=eta, bits=M.FREE_SLIP, mask=M.dirichlet_mask(m, m, m, M.FREE_SLIP))
    x = np.random.default_rng(4).uniform(-1.0, 1.0, size=c.size)
    op = make_op(case)
    assert op.geometry_mode == GEOM_AFFINE
    y = torch.empty(x.size, dtype=torch.float64, device="cuda")
    op.mult(T(x), y)
    y64 = host(y)
    reference_kernels.setup((m, m, m), c, eta)
    ref = matmult_a11(lambda v: reference_kernels.a11_raw(v, "avx"), x, case["mask"])
    assert rel(y64, ref) <= TOL64
    op32 = make_op(case, prec=PREC_F32)
    y32 = torch.empty(x.size, dtype=torch.float32, device="cuda")
    op32.mult(T(x, torch.float32), y32)
    assert rel(host(y32), y64) <= TOL32


@pytest.mark.parametrize("dims", [(13, 7, 5), (1, 1, 1), (9, 5, 3), (8, 4, 2), (6, 4, 17), (11, 3, 8)])
@pytest.mark.parametrize("geom", [GEOM_GENERAL, GEOM_AFFINE])
def test_fp32_ragged(cuda, dims, geom):
    """The FP32 A11 kernels on ragged meshes (bricks cut by the mesh edges),
    affine and general geometry, in the MatMult and the raw (y +=) forms,
    against the FP64 operator."""
    mx, my, mz = dims
    c = M.uniform_coords(mx, my, mz, hi=(1.0, 2.0, 0.5))
    if geom == GEOM_GENERAL:
        c = M.perturb_interior(c, mx, my, mz, frac=0.15, seed=sum(dims))
    eta = 10 ** np.random.default_rng(1).uniform(-1, 1, size=(mx * my * mz, 27))
    case = dict(dims=dims, coords=c, eta=eta, bits=M.FREE_SLIP)
    op64, op32 = make_op(case), make_op(case, prec=PREC_F32)
    assert op32.geometry_mode == geom and op64.geometry_mode == geom
    x = np.random.default_rng(2).uniform(-1, 1, size=c.size)
    y64 = torch.empty(x.size, dtype=torch.float64, device="cuda")
    y32 = torch.empty(x.size, dtype=torch.float32, device="cuda")
    op64.mult(T(x), y64)
    op32.mult(T(x, torch.float32), y32)
    assert rel(host(y32), host(y64)) <= TOL32
    y0 = np.random.default_rng(3).uniform(-1, 1, size=x.size)  # y += A x keeps the old y
    z64, z32 = T(y0), T(y0, torch.float32)
    op64.spmv(T(x), z64)
    op32.spmv(T(x, torch.float32), z32)
    assert rel(host(z32), host(z64)) <= TOL32


@pytest.mark.parametrize("geom,prec", [(GEOM_AFFINE, PREC_F64), (GEOM_GENERAL, PREC_F64), (GEOM_AFFINE, PREC_F32),
                                       (GEOM_GENERAL, PREC_F32)])
def test_grouped_mult_equals_member_mults(cuda, geom, prec):
    """p3d_a11_mult_grouped: five operators of one mesh shape with different
    coefficients applied in one launch give each member's own MatMult, and a
    member of another shape is refused."""
    import ctypes as C

    from ptatin3d_b200 import _lib
    dims = (9, 6, 7)
    dt = torch.float64 if prec == PREC_F64 else torch.float32
    ops, xs, ys, refs = [], [], [], []
    for k in range(5):
        c = M.uniform_coords(*dims)
        if geom == GEOM_GENERAL:
            c = M.perturb_interior(c, *dims, frac=0.15, seed=k)
        eta = 10 ** np.random.default_rng(k).uniform(-1, 1, size=(int(np.prod(dims)), 27))
        op = make_op(dict(dims=dims, coords=c, eta=eta, bits=M.FREE_SLIP), prec=prec)
        assert op.geometry_mode == geom
        x = T(np.random.default_rng(10 + k).uniform(-1, 1, size=c.size), dt)
        r = torch.empty_like(x)
        op.mult(x, r)
        ops.append(op); xs.append(x); ys.append(torch.full_like(x, float("nan"))); refs.append(r)
    P = C.c_void_p * 5
    rc = _lib.lib().p3d_a11_mult_grouped(P(*[o.h.value for o in ops]), P(*[x.data_ptr() for x in xs]),
                                         P(*[y.data_ptr() for y in ys]), 5, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize()
    for y, r in zip(ys, refs):
        assert rel(host(y), host(r)) <= (1e-14 if prec == PREC_F64 else 1e-6)
    other = make_op(dict(dims=(9, 6, 8), coords=M.uniform_coords(9, 6, 8), eta=np.ones((9 * 6 * 8, 27)), bits=M.FREE_SLIP),
                    prec=prec)
    P2 = C.c_void_p * 2
    x2 = T(np.zeros(other.n_velocity), dt)
    rc = _lib.lib().p3d_a11_mult_grouped(P2(ops[0].h.value, other.h.value), P2(xs[0].data_ptr(), x2.data_ptr()),
                                         P2(ys[0].data_ptr(), x2.data_ptr()), 2, None)
    assert rc == _lib.P3D_ERR_ARG
