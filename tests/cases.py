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
