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
