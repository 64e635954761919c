"""The CPU restatement of the solver (oracle/cpu_solver.py, the CPU solve
baseline of bench.py) solves the oracle's assembled Stokes system, and on the
GPU it takes the same path as the device solver."""
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
