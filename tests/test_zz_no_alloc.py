"""p3d_a11_apply_host_noalloc: the A11 host-buffer apply for callers that may
not allocate device memory (its x/y staging lives in a fixed static device
array instead of buffers obtained from cudaMalloc).

Checked through the C ABI against p3d_a11_apply_host, which computes the
same apply with allocated staging, and against the oracle's MatMult, on two
calls in a row: the static array keeps the previous call's contents, so the
second call also checks that y starts from zero.  Three meshes cover the
kernel paths the entry point can take: a deformed 16^3 mesh (per-point
Jacobians), an undeformed 16^3 mesh (the affine kernel) and a rank's owned
block inside a ghosted lattice (the size limit counts the ghosted lattice).
Collected last (file name) so a failure here does not hide the rest of the
suite.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Restatement, matmult_a11
from ptatin3d_b200 import _lib
from ptatin3d_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _whole(m, deform, seed):
    """A whole m^3 mesh with free slip on every face; oracle MatMult of x."""
    d = _lib.MeshDesc()
    assert _lib.lib().p3d_mesh_desc_whole(m, m, m, M.FREE_SLIP, C.byref(d)) == 0
    c = M.uniform_coords(m, m, m)
    if deform:
        c = M.perturb_interior(c, m, m, m, frac=deform, seed=seed)
    eta = M.sinker_eta(M.qp_coords(c, m, m, m), [[0.4, 0.5, 0.6]], 0.3, 1.0, 50.0)
    mask = M.dirichlet_mask(m, m, m, M.FREE_SLIP)
    R = Restatement()

    def oracle(x):
        return matmult_a11(lambda v: R.a11_raw((m, m, m), c, eta.reshape(-1), v), x, mask)

    return d, c, np.ascontiguousarray(eta), oracle, _lib.BC_MATMULT


def _ghosted(seed):
    """An interior rank's 4x3x5 owned block inside a lattice with 2 ghost
    nodes on some sides (PETSc local vectors); raw element apply."""
    mx, my, mz = 4, 3, 5
    lo, hi = (2, 0, 2), (2, 2, 0)
    gx, gy, gz = (2 * m + 1 + a + b for m, a, b in zip((mx, my, mz), lo, hi))
    c = M.uniform_coords(gx // 2, gy // 2, gz // 2).reshape(gz, gy, gx, 3).copy()
    owned = (slice(lo[2], lo[2] + 2 * mz + 1), slice(lo[1], lo[1] + 2 * my + 1), slice(lo[0], lo[0] + 2 * mx + 1))
    c_loc = M.perturb_interior(M.uniform_coords(mx, my, mz), mx, my, mz, frac=0.15, seed=seed)
    c[owned] = c_loc.reshape(2 * mz + 1, 2 * my + 1, 2 * mx + 1, 3)
    eta = 10 ** np.random.default_rng(seed).uniform(-1, 1, size=(mx * my * mz, 27))
    d = _lib.MeshDesc()
    assert _lib.lib().p3d_mesh_desc_whole(mx, my, mz, M.FREE_SLIP, C.byref(d)) == 0
    d.gx, d.gy, d.gz = gx, gy, gz
    d.ox, d.oy, d.oz = lo
    d.global_faces = 0
    R = Restatement()

    def oracle(x):
        y = np.zeros((gz, gy, gx, 3))
        xl = x.reshape(gz, gy, gx, 3)[owned].reshape(-1)
        y[owned] = R.a11_raw((mx, my, mz), c_loc, eta.reshape(-1), xl).reshape(2 * mz + 1, 2 * my + 1, 2 * mx + 1, 3)
        return y.reshape(-1)

    return d, c.reshape(-1), np.ascontiguousarray(eta), oracle, _lib.BC_NONE


CASES = {
    "deformed_16": lambda: _whole(16, 0.15, 3),  # 3 * 33^3 = 107,811 dofs: exactly the static limit
    "affine_16": lambda: _whole(16, 0.0, 3),
    "ghosted": lambda: _ghosted(5),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_noalloc_matches_allocating_apply(cuda, name):
    d, c, eta, oracle, bc = CASES[name]()
    L = _lib.lib()
    h = C.c_void_p()
    _lib.check(L.p3d_op_create(C.byref(d), _lib.PREC_F64, 0, C.byref(h)))
    try:
        _lib.check(L.p3d_op_set_coefficients(h, _p(np.ascontiguousarray(c)), _p(eta), 0))
        _lib.check(L.p3d_op_set_bc_mode(h, bc))
        mode = C.c_int()
        _lib.check(L.p3d_op_geometry_mode(h, C.byref(mode)))
        assert mode.value == (_lib.GEOM_AFFINE if name == "affine_16" else _lib.GEOM_GENERAL)
        n = 3 * d.gx * d.gy * d.gz
        assert n <= _lib.NOALLOC_MAX_DOFS
        rng = np.random.default_rng(11)
        for call in range(2):
            x = rng.uniform(-1.0, 1.0, size=n)
            y_ref = np.empty(n)
            y_na = np.full(n, np.nan)
            _lib.check(L.p3d_a11_apply_host(h, _p(x), _p(y_ref)))
            _lib.check(L.p3d_a11_apply_host_noalloc(h, _p(x), _p(y_na)))
            y_or = oracle(x)
            assert np.linalg.norm(y_na - y_ref) <= TOL * np.linalg.norm(y_ref), (name, call)
            assert np.linalg.norm(y_na - y_or) <= TOL * np.linalg.norm(y_or), (name, call)
    finally:
        L.p3d_op_destroy(h)


def test_noalloc_rejects_meshes_above_the_limit(cuda):
    L = _lib.lib()
    d = _lib.MeshDesc()
    assert L.p3d_mesh_desc_whole(17, 17, 17, M.FREE_SLIP, C.byref(d)) == 0  # 3 * 35^3 = 128,625 dofs
    h = C.c_void_p()
    _lib.check(L.p3d_op_create(C.byref(d), _lib.PREC_F64, 0, C.byref(h)))
    try:
        c = M.uniform_coords(17, 17, 17)
        eta = np.ones((17 ** 3, 27))
        _lib.check(L.p3d_op_set_coefficients(h, _p(c), _p(eta), 0))
        n = c.size
        x, y = np.zeros(n), np.zeros(n)
        rc = L.p3d_a11_apply_host_noalloc(h, _p(x), _p(y))
        assert rc == _lib.P3D_ERR_ARG
        assert b"static limit" in L.p3d_last_error()
    finally:
        L.p3d_op_destroy(h)
