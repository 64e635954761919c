"""The material-point -> Gauss-point projections of the reference's rheology
update (src/rheology.c:150-185): the numpy restatement (oracle.marker_project)
and the reference's own compiled functions (oracle/_ref) against the committed
golden vectors, which tests/golden/make_marker_golden.py made with the
reference's functions."""
import os

import numpy as np
import pytest

from oracle.oracle import marker_project

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "markers_3x2x4.npz")
TYPES = (0, 10, 20, 1)


def gold():
    return np.load(GOLD)


def close(a, b, rtol):
    """Equal NaN positions, elsewhere |a - b| <= rtol |b|."""
    a, b = np.asarray(a), np.asarray(b)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    m = ~np.isnan(b)
    return bool(np.all(np.abs(a[m] - b[m]) <= rtol * np.abs(b[m]) + 1e-300))


@pytest.mark.parametrize("case", ["dense", "sparse"])
@pytest.mark.parametrize("ptype", TYPES)
def test_restatement_matches_golden(case, ptype):
    g = gold()
    dims = tuple(int(v) for v in g["dims"])
    eq, rq = marker_project(dims, ptype, g[f"{case}_wil"], g[f"{case}_xi"], g[f"{case}_eta"], g[f"{case}_rho"])
    assert close(eq, g[f"{case}_{ptype}_eta_q"], 1e-14)
    assert close(rq, g[f"{case}_{ptype}_rho_q"], 1e-14)


def test_restatement_one2one_and_null():
    g = gold()
    dims = tuple(int(v) for v in g["dims"])
    eq, rq = marker_project(dims, 4, g["one2one_wil"], None, g["one2one_eta"], g["one2one_rho"])
    assert np.array_equal(eq, g["one2one_eta_q"]) and np.array_equal(rq, g["one2one_rho_q"])
    e0, r0 = np.full(eq.size, 3.0), np.full(eq.size, 5.0)
    eq, rq = marker_project(dims, -1, g["dense_wil"], g["dense_xi"], g["dense_eta"], g["dense_rho"], e0, r0)
    assert np.array_equal(eq, e0) and np.array_equal(rq, r0)


def test_sparse_case_has_empty_elements():
    """The sparse golden covers the reference's edge cases: elements without
    markers (P0: 0/0) next to elements with them."""
    g = gold()
    assert np.isnan(g["sparse_0_eta_q"]).any() and not np.isnan(g["sparse_0_eta_q"]).all()
    assert np.isfinite(g["sparse_1_eta_q"]).all()


@pytest.mark.parametrize("case", ["dense", "sparse"])
def test_reference_functions_reproduce_golden(reference_kernels, case):
    from ptatin3d_b200 import mesh as M
    g = gold()
    dims = tuple(int(v) for v in g["dims"])
    nel = dims[0] * dims[1] * dims[2]
    reference_kernels.setup(dims, M.uniform_coords(*dims), np.ones(27 * nel))
    for t in TYPES:
        eq, rq = reference_kernels.marker_project(t, g[f"{case}_wil"], g[f"{case}_xi"], g[f"{case}_eta"],
                                                  g[f"{case}_rho"])
        assert close(eq, g[f"{case}_{t}_eta_q"], 0.0) and close(rq, g[f"{case}_{t}_rho_q"], 0.0)


def test_restatement_vs_reference_random(reference_kernels):
    """A larger random case, markers per element uneven, viscosity over 6 decades."""
    from ptatin3d_b200 import mesh as M
    dims = (5, 4, 6)
    nel = dims[0] * dims[1] * dims[2]
    rng = np.random.default_rng(5)
    n = 15 * nel
    wil = rng.integers(0, nel, size=n).astype(np.int32)
    xi = rng.uniform(-1, 1, size=(n, 3))
    eta, rho = 10.0 ** rng.uniform(-3, 3, size=n), rng.uniform(0.9, 1.1, size=n)
    reference_kernels.setup(dims, M.uniform_coords(*dims), np.ones(27 * nel))
    for t in TYPES:
        er, rr = reference_kernels.marker_project(t, wil, xi, eta, rho)
        en, rn = marker_project(dims, t, wil, xi, eta, rho)
        assert close(en, er, 1e-13) and close(rn, rr, 1e-13)


def test_restated_type1_hierarchy_starts_from_marker_nodes(restatement):
    """The type-1 hierarchy restricts the markers' nodal field; when that field
    is the nodal projection of the Gauss-point values, it equals the hierarchy
    built from those values."""
    dims = (8, 8, 8)
    rng = np.random.default_rng(3)
    nel = 512
    n = 10 * nel
    wil = rng.integers(0, nel, size=n).astype(np.int32)
    xi = rng.uniform(-1, 1, size=(n, 3))
    eta, rho = 10.0 ** rng.uniform(-2, 2, size=n), np.ones(n)
    eq, _, v = marker_project(dims, 1, wil, xi, eta, rho, nodal=True)
    assert v.size == 17 ** 3 and np.all(v > 0)
    lv = restatement.eta_hierarchy_from_nodes(dims, eq, v, 3)
    assert [a.size for a in lv] == [27 * 512, 27 * 64, 27 * 8]
    assert np.array_equal(lv[0], eq)
    # started from the Gauss-point projection, the two hierarchies agree
    qp = restatement.eta_hierarchy(dims, eq, 3)
    import ctypes as C
    from oracle.oracle import _dp, _p
    restatement.L.o_eta_project_nodes.argtypes = [C.c_int] * 3 + [_dp] * 2
    vq = np.zeros(17 ** 3)
    restatement.L.o_eta_project_nodes(8, 8, 8, _p(np.ascontiguousarray(eq)), _p(vq))
    for a, b in zip(restatement.eta_hierarchy_from_nodes(dims, eq, vq, 3), qp):
        assert np.allclose(a, b, rtol=1e-14, atol=0)
