"""Shared construction of the operator test cases (meshes, viscosity, vectors)."""
import numpy as np

from ptatin3d_b200 import mesh as M


def bump_case(mx, my, mz, eta_kind="one", seed=0):
    """Viscous-sinker operator test mesh: unit cube + Gaussian bump on y-max,
    free-slip/free-surface boundary, reference test vectors."""
    c = M.gaussian_bump_ymax(M.uniform_coords(mx, my, mz), mx, my, mz)
    nel = mx * my * mz
    if eta_kind == "one":
        eta = np.ones((nel, 27))
    else:
        rng = np.random.default_rng(seed)
        eta = 10.0 ** rng.uniform(-2, 2, size=(nel, 27))
    bits = M.FREE_SLIP_FREE_SURFACE
    return dict(dims=(mx, my, mz), coords=c, eta=eta, bits=bits, mask=M.dirichlet_mask(mx, my, mz, bits),
                x=M.test_vector_velocity(c), p=M.test_vector_pressure(mx, my, mz))


def sinker_case(m, seed=1, nsph=8, radius=0.1, eta1=1e3, deform=0.0):
    """Unit cube, eta = 1 outside / eta1 inside seeded spheres, random x, free slip on all faces."""
    c = M.uniform_coords(m, m, m)
    if deform:
        c = M.perturb_interior(c, m, m, m, frac=deform, seed=seed)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(nsph, seed, radius)
    eta = M.sinker_eta(qp, cen, r, 1.0, eta1)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=c.size)
    p = rng.uniform(-1.0, 1.0, size=4 * m ** 3)
    bits = M.FREE_SLIP
    return dict(dims=(m, m, m), coords=c, eta=eta, bits=bits, mask=M.dirichlet_mask(m, m, m, bits), x=x, p=p)


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solcx_case(mx, my, mz, eta0, eta1, xc=0.5, n=2):
    """The reference's SolCx verification model (src/models/analytics_vv/analytics_vv.c):
    unit cube, free slip on all six faces (:68-83), gravity (0, -1, 0) (:115-125),
    markers on the Gauss points mapped one to one (projection type 4), eta = eta0
    for x <= xc else eta1 and rho = -cos(pi x) sin(n pi y) at each point (:221-257)."""
    c = M.uniform_coords(mx, my, mz)
    qp = M.qp_coords(c, mx, my, mz)
    x, y = qp[..., 0], qp[..., 1]
    eta = np.where(x <= xc, eta0, eta1)
    rho = -np.cos(np.pi * x) * np.sin(n * np.pi * y)
    bits = M.FREE_SLIP
    return dict(dims=(mx, my, mz), coords=c, eta=eta, rho=rho, bits=bits, mask=M.dirichlet_mask(mx, my, mz, bits),
                g=(0.0, -1.0, 0.0))


def _q2_1d(x):
    return np.stack([0.5 * x * (x - 1.0), 1.0 - x * x, 0.5 * x * (x + 1.0)], axis=-1)


def sinker_markers(case, eta0=1.0, eta1=10.0, rho0=0.0, rho1=1.0, per_dir=2):
    """Material points of the reference's viscous-sinker operator tests on the
    mesh of `case`: per_dir^3 markers per element on the lattice
    xi = -1 + (2/per_dir)(i + 1/2) (SwarmMPntStd_CoordAssignment_LatticeLayout3d,
    src/material_point_std_utils.c:100-200; 2^3 by default, src/ptatin3d.c:473,
    the tests set -lattice_layout_perturb 0), placed through the element's Q2
    map, eta1 / -rho1 inside the sphere of diameter 0.5 about the box centre and
    eta0 / -rho0 outside (src/models/viscous_sinker/model_viscous_sinker_ops.c:
    70-85, 755-770).  Returns (wil, xi [n,3], eta, rho)."""
    mx, my, mz = case["dims"]
    c = np.asarray(case["coords"]).reshape(-1, 3)
    nx, ny = 2 * mx + 1, 2 * my + 1
    s = -1.0 + (2.0 / per_dir) * (np.arange(per_dir) + 0.5)
    xi = np.array([(s[i], s[j], s[k]) for k in range(per_dir) for j in range(per_dir) for i in range(per_dir)])
    Ni = (_q2_1d(xi[:, 0])[:, None, None, :] * _q2_1d(xi[:, 1])[:, None, :, None]
          * _q2_1d(xi[:, 2])[:, :, None, None]).reshape(len(xi), 27)
    e = np.arange(mx * my * mz)
    ex, ey, ez = e % mx, (e // mx) % my, e // (mx * my)
    n = np.arange(27)
    nodes = (2 * ex[:, None] + n % 3) + nx * ((2 * ey[:, None] + (n // 3) % 3) + ny * (2 * ez[:, None] + n // 9))
    pos = np.einsum("pn,enk->epk", Ni, c[nodes]).reshape(-1, 3)
    inside = (((pos - 0.5) / 0.25) ** 2).sum(axis=1) < 1.0
    wil = np.repeat(e, len(xi)).astype(np.int32)
    return (wil, np.tile(xi, (len(e), 1)), np.where(inside, eta1, eta0), np.where(inside, -rho1, -rho0))
