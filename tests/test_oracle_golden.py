"""Pin the CPU oracle (restatement and the reference's own compiled kernels)
against the known answers printed by the reference's operator tests
(tests/integration/operator/**/expected, extracted into
tests/golden/reference_expected.json by tests/golden/make_golden.py).

Exact pins: A12 and A21 do not depend on viscosity; A11 and diag(A11) are
pinned where the test's viscosity field is uniform (default sinker with
eta1 = 1, and the 1x1x3 mesh whose Gauss points never sample the inclusion),
and, for the eta1 = 10 sinker, with the Gauss-point viscosity the reference
computes from its material points: a 2^3 marker lattice per element and the
Q1 projection (tests/cases.py:sinker_markers, projection type 1).
The reference harness compares at 1e-13; the values are printed with 9
significant digits, so agreement is checked to 5e-9 relative.
"""
import json
import math
import os

import numpy as np
import pytest

from cases import bump_case, sinker_markers
from oracle.oracle import get_diagonal, marker_project, matmult_a11, matmult_a12, matmult_a21

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_expected.json")))


def _pins():
    out = []
    for name, rec in GOLD.items():
        dims = (rec["mx"], rec["my"], rec["mz"])
        uniform_eta = rec["eta1"] == 1.0 or dims == (1, 1, 3)
        for op in ("A21", "A12") + (("A11", "diagA11") if uniform_eta else ()):
            if op in rec:
                out.append(pytest.param(name, op, dims, float(rec[op]), id=f"{name}-{op}"))
    return out


def _check(val, gold):
    if math.isnan(gold):
        assert math.isnan(val)
    else:
        assert abs(val - gold) <= 5e-9 * abs(gold), (val, gold)


def _yy(impl, op, case):
    d, c, eta, mask = case["dims"], case["coords"], case["eta"], case["mask"]
    if op == "A11":
        y = matmult_a11(lambda v: impl["a11"](v), case["x"], mask)
    elif op == "diagA11":
        y = get_diagonal(impl["diag"], mask)
    elif op == "A21":
        y = matmult_a21(impl["a21"], case["x"], mask)
    else:
        y = matmult_a12(impl["a12"], case["p"], mask)
    return float(y @ y)


@pytest.mark.parametrize("name,op,dims,gold", _pins())
def test_restatement_matches_reference_expected(restatement, name, op, dims, gold):
    case = bump_case(*dims)
    d, c, eta = case["dims"], case["coords"], case["eta"].reshape(-1)
    impl = {"a11": lambda v: restatement.a11_raw(d, c, eta, v), "diag": lambda: restatement.diag_raw(d, c, eta),
            "a21": lambda v: restatement.a21_raw(d, c, v), "a12": lambda v: restatement.a12_raw(d, c, v)}
    _check(_yy(impl, op, case), gold)


@pytest.mark.parametrize("name,op,dims,gold", [p for p in _pins() if p.values[2][0] * p.values[2][1] * p.values[2][2] <= 1500])
def test_reference_kernels_match_reference_expected(reference_kernels, name, op, dims, gold):
    case = bump_case(*dims)
    reference_kernels.setup(case["dims"], case["coords"], case["eta"])
    impl = {"a11": lambda v: reference_kernels.a11_raw(v, "tensor"), "diag": reference_kernels.diag_raw,
            "a21": reference_kernels.a21_raw, "a12": reference_kernels.a12_raw}
    _check(_yy(impl, op, case), gold)


def _marker_pins(max_nel=None):
    out = []
    for name, rec in GOLD.items():
        dims = (rec["mx"], rec["my"], rec["mz"])
        if rec["eta1"] == 1.0 or (max_nel and dims[0] * dims[1] * dims[2] > max_nel):
            continue
        for op in ("A11", "diagA11"):
            out.append(pytest.param(name, op, dims, rec["eta1"], float(rec[op]), id=f"{name}-{op}-markers"))
    return out


@pytest.mark.parametrize("name,op,dims,eta1,gold", _marker_pins())
def test_restatement_with_marker_viscosity_matches_reference_expected(restatement, name, op, dims, eta1, gold):
    """eta1 = 10 sinker: markers -> Q1 projection (numpy restatement) -> A11 / diag(A11)."""
    case = bump_case(*dims)
    wil, xi, eta_p, rho_p = sinker_markers(case, eta1=eta1)
    eta, _ = marker_project(dims, 1, wil, xi, eta_p, rho_p)
    d, c = case["dims"], case["coords"]
    impl = {"a11": lambda v: restatement.a11_raw(d, c, eta, v), "diag": lambda: restatement.diag_raw(d, c, eta)}
    _check(_yy(impl, op, case), gold)


@pytest.mark.parametrize("name,op,dims,eta1,gold", _marker_pins(max_nel=1500))
def test_reference_projection_and_kernels_match_reference_expected(reference_kernels, name, op, dims, eta1, gold):
    """The same with the reference's own compiled projection and kernels throughout."""
    case = bump_case(*dims)
    wil, xi, eta_p, rho_p = sinker_markers(case, eta1=eta1)
    nel = dims[0] * dims[1] * dims[2]
    reference_kernels.setup(dims, case["coords"], np.ones(27 * nel))
    eta, _ = reference_kernels.marker_project(1, wil, xi, eta_p, rho_p)
    reference_kernels.setup(dims, case["coords"], eta)
    impl = {"a11": lambda v: reference_kernels.a11_raw(v, "tensor"), "diag": reference_kernels.diag_raw}
    _check(_yy(impl, op, case), gold)


@pytest.mark.parametrize("variant", ["tensor", "avx", "ref"])
def test_restatement_vs_reference_kernels_random(restatement, reference_kernels, variant):
    """Random viscosity (4 decades), deformed mesh: every reference backend vs the restatement."""
    case = bump_case(4, 3, 5, eta_kind="random", seed=3)
    d, c, eta = case["dims"], case["coords"], case["eta"]
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=c.size)
    p = rng.uniform(-1, 1, size=4 * 60)
    reference_kernels.setup(d, c, eta)
    y0 = restatement.a11_raw(d, c, eta.reshape(-1), x)
    y1 = reference_kernels.a11_raw(x, variant)
    assert np.linalg.norm(y0 - y1) <= 1e-13 * np.linalg.norm(y1)
    if variant == "tensor":
        for a, b in [(restatement.diag_raw(d, c, eta.reshape(-1)), reference_kernels.diag_raw()),
                     (restatement.a12_raw(d, c, p), reference_kernels.a12_raw(p)),
                     (restatement.a21_raw(d, c, x), reference_kernels.a21_raw(x))]:
            assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


def test_reference_avx_a12_and_fused_operator(restatement, reference_kernels):
    """The AVX back end's A12 and fused [A11 A12; A21 0] (what the CPU solve
    baseline calls) against the restatement."""
    case = bump_case(4, 3, 5, eta_kind="random", seed=3)
    d, c, eta = case["dims"], case["coords"], case["eta"]
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, size=c.size)
    p = rng.uniform(-1, 1, size=4 * 60)
    reference_kernels.setup(d, c, eta)
    ya12 = reference_kernels.a12_avx_raw(p)
    ref12 = restatement.a12_raw(d, c, p)
    assert np.linalg.norm(ya12 - ref12) <= 1e-13 * np.linalg.norm(ref12)
    yu, yp = reference_kernels.stokes_avx_raw(x, p)
    ref_u = restatement.a11_raw(d, c, eta.reshape(-1), x) + ref12
    ref_p = restatement.a21_raw(d, c, x)
    assert np.linalg.norm(yu - ref_u) <= 1e-13 * np.linalg.norm(ref_u)
    assert np.linalg.norm(yp - ref_p) <= 1e-13 * np.linalg.norm(ref_p)


def test_element_matrix_consistent_with_apply(restatement):
    """The 81x81 element matrix reproduces the matrix-free element apply."""
    case = bump_case(1, 1, 1, eta_kind="random", seed=7)
    c, eta = case["coords"], case["eta"].reshape(-1)
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, size=c.size)
    K = restatement.element_matrix(c.reshape(27, 3), eta)
    y = restatement.a11_raw((1, 1, 1), c, eta, x)
    assert np.allclose(K @ x, y, rtol=1e-12, atol=1e-12 * np.abs(y).max())
    assert np.allclose(K, K.T, atol=1e-12 * np.abs(K).max())


def test_transfer_adjoint(restatement):
    rng = np.random.default_rng(2)
    cn = (3, 4, 2)
    xc = rng.standard_normal(3 * 24)
    xf = rng.standard_normal(3 * 5 * 7 * 3)
    assert abs(restatement.prolong(cn, 3, xc) @ xf - xc @ restatement.restrict(cn, 3, xf)) < 1e-12
    # prolongation reproduces trilinear fields exactly
    I, J, K = np.meshgrid(np.arange(3), np.arange(4), np.arange(2), indexing="ij")
    lin = (1 + 2 * I + 3 * J - K).transpose(2, 1, 0).reshape(-1)
    f = restatement.prolong(cn, 1, lin)
    Fi, Fj, Fk = np.meshgrid(np.arange(5) / 2, np.arange(7) / 2, np.arange(3) / 2, indexing="ij")
    assert np.allclose(f, (1 + 2 * Fi + 3 * Fj - Fk).transpose(2, 1, 0).reshape(-1))


def test_q1_coefficient_hierarchy_restatement(restatement):
    """The oracle's Q1 viscosity hierarchy: constants are reproduced exactly,
    values stay inside the fine range (clamping), and the nodal projection of
    an element-wise field is its weighted average."""
    import numpy as np
    m = 4
    eta = np.full((m ** 3, 27), 3.5)
    for e in restatement.eta_hierarchy((m, m, m), eta, 3):
        assert np.allclose(e, 3.5, rtol=0, atol=1e-14)
    rng = np.random.default_rng(1)
    eta = 10.0 ** rng.uniform(-2, 2, size=(m ** 3, 27))
    levels = restatement.eta_hierarchy((m, m, m), eta, 3)
    assert [lv.size for lv in levels] == [27 * 64, 27 * 8, 27]
    for e in levels[1:]:
        assert e.min() >= eta.min() - 1e-12 and e.max() <= eta.max() + 1e-12


def test_loworder_golden_is_the_reference_kernel(reference_kernels):
    """The committed low-order golden vectors are reproduced by the reference's compiled kernel."""
    import os
    import numpy as np
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "loworder_4x3x5.npz"))
    reference_kernels.setup(tuple(int(v) for v in g["dims"]), g["coords"], g["eta"])
    y = reference_kernels.a11_raw(g["x"], "loworder")
    assert np.linalg.norm(y - g["y"]) <= 1e-14 * np.linalg.norm(g["y"])
