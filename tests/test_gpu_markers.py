"""Material points -> Gauss points on the device (p3d_marker_project) against
the reference's own projections: the committed golden vectors (made by the
reference's compiled functions) and the numpy restatement on larger meshes.
Tolerance 1e-12 relative (FP64; the device sums markers in atomic order)."""
import os

import numpy as np
import pytest

from oracle.oracle import marker_project

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "markers_3x2x4.npz")
TYPES = (0, 10, 20, 1)


def close(a, b, rtol):
    a, b = np.asarray(a).reshape(-1), np.asarray(b).reshape(-1)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    m = ~np.isnan(b)
    return bool(np.all(np.abs(a[m] - b[m]) <= rtol * np.abs(b[m]) + 1e-300))


def device_markers(cuda, wil, xi, eta, rho):
    import torch
    t = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)
    return (t(wil, torch.int32), None if xi is None else t(np.asarray(xi).reshape(-1, 3), torch.float64),
            t(eta, torch.float64), t(rho, torch.float64))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["dense", "sparse"])
@pytest.mark.parametrize("ptype", TYPES)
def test_device_projection_matches_golden(cuda, case, ptype):
    from ptatin3d_b200.markers import update_gauss_properties
    g = np.load(GOLD)
    dims = tuple(int(v) for v in g["dims"])
    w, x, e, r = device_markers(cuda, g[f"{case}_wil"], g[f"{case}_xi"], g[f"{case}_eta"], g[f"{case}_rho"])
    eq, rq = update_gauss_properties(dims, ptype, w, x, e, r)
    assert close(eq.cpu().numpy(), g[f"{case}_{ptype}_eta_q"], 1e-12)
    assert close(rq.cpu().numpy(), g[f"{case}_{ptype}_rho_q"], 1e-12)


@pytest.mark.gpu
def test_device_one2one_and_null(cuda):
    import torch
    from ptatin3d_b200.markers import PROJ_NULL, PROJ_ONE2ONE, update_gauss_properties
    g = np.load(GOLD)
    dims = tuple(int(v) for v in g["dims"])
    w, _, e, r = device_markers(cuda, g["one2one_wil"], None, g["one2one_eta"], g["one2one_rho"])
    eq, rq = update_gauss_properties(dims, PROJ_ONE2ONE, w, None, e, r)
    assert np.array_equal(eq.cpu().numpy().reshape(-1), g["one2one_eta_q"])
    assert np.array_equal(rq.cpu().numpy().reshape(-1), g["one2one_rho_q"])
    e0 = torch.full_like(eq, 3.0)
    r0 = torch.full_like(rq, 5.0)
    w, x, e, r = device_markers(cuda, g["dense_wil"], g["dense_xi"], g["dense_eta"], g["dense_rho"])
    update_gauss_properties(dims, PROJ_NULL, w, x, e, r, e0, r0)
    assert bool((e0 == 3.0).all()) and bool((r0 == 5.0).all())


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 16, 16), (13, 7, 9)])
def test_device_projection_vs_restatement(cuda, dims):
    """Uneven marker counts per element, viscosity over 6 decades, some markers
    outside the mesh (element index -1 or >= nel: skipped on the device, left
    out of the restatement's input)."""
    from ptatin3d_b200.markers import update_gauss_properties
    nel = dims[0] * dims[1] * dims[2]
    rng = np.random.default_rng(9)
    n = 12 * nel
    wil = rng.integers(0, nel, size=n).astype(np.int32)
    xi = rng.uniform(-1, 1, size=(n, 3))
    eta, rho = 10.0 ** rng.uniform(-3, 3, size=n), rng.uniform(0.9, 1.1, size=n)
    bad = rng.choice(n, size=50, replace=False)
    wil_dev = wil.copy()
    wil_dev[bad[:25]] = -1
    wil_dev[bad[25:]] = nel + 7
    keep = np.ones(n, dtype=bool)
    keep[bad] = False
    w, x, e, r = device_markers(cuda, wil_dev, xi, eta, rho)
    for t in TYPES:
        eq, rq = update_gauss_properties(dims, t, w, x, e, r)
        en, rn = marker_project(dims, t, wil[keep], xi[keep], eta[keep], rho[keep])
        assert close(eq.cpu().numpy(), en, 1e-12), t
        assert close(rq.cpu().numpy(), rn, 1e-12), t


@pytest.mark.gpu
def test_device_projection_errors(cuda):
    import torch
    from ptatin3d_b200 import P3DError
    from ptatin3d_b200.markers import PROJ_ONE2ONE, update_gauss_properties
    w, x, e, r = device_markers(cuda, np.zeros(5, np.int32), np.zeros((5, 3)), np.ones(5), np.ones(5))
    with pytest.raises(P3DError):
        update_gauss_properties((2, 2, 2), 3, w, x, e, r)  # P1 projection: not a type the reference supports
    with pytest.raises(P3DError):
        update_gauss_properties((2, 2, 2), PROJ_ONE2ONE, w, x, e, r)  # needs 27 markers per element
    torch.cuda.synchronize()
