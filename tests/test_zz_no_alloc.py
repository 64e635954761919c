"""p3d_a11_apply_host_noalloc: the A11 host-buffer apply for callers that may
not allocate device memory (its x/y staging lives in a fixed static device
array instead of buffers obtained from cudaMalloc).

Checked through the C ABI against p3d_a11_apply_host, which computes the
same apply with allocated staging, on two calls in a row: the static array
keeps the previous call's contents, so the second call also checks that y
starts from zero.  Collected last (file name) so a failure here does not hide
the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from ptatin3d_b200 import _lib
from ptatin3d_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _op(m, seed):
    import torch  # noqa: F401  (initialises the CUDA context the library shares)
    L = _lib.lib()
    d = _lib.MeshDesc()
    assert L.p3d_mesh_desc_whole(m, m, m, M.FREE_SLIP, C.byref(d)) == 0
    h = C.c_void_p()
    _lib.check(L.p3d_op_create(C.byref(d), _lib.PREC_F64, 0, C.byref(h)))
    c = M.perturb_interior(M.uniform_coords(m, m, m), m, m, m, frac=0.15, seed=seed)
    eta = M.sinker_eta(M.qp_coords(c, m, m, m), [[0.4, 0.5, 0.6]], 0.3, 1.0, 50.0)
    _lib.check(L.p3d_op_set_coefficients(h, c.ctypes.data_as(C.c_void_p), np.ascontiguousarray(eta).ctypes.data_as(C.c_void_p), 0))
    return L, h, c.size


def test_noalloc_matches_allocating_apply(cuda):
    L, h, n = _op(16, seed=3)  # the largest mesh the static staging holds
    assert n == 107811  # exactly the static limit
    rng = np.random.default_rng(11)
    try:
        for call in range(2):
            x = rng.uniform(-1.0, 1.0, size=n)
            y_ref = np.empty(n)
            y_na = np.full(n, np.nan)
            _lib.check(L.p3d_a11_apply_host(h, x.ctypes.data_as(C.c_void_p), y_ref.ctypes.data_as(C.c_void_p)))
            _lib.check(L.p3d_a11_apply_host_noalloc(h, x.ctypes.data_as(C.c_void_p), y_na.ctypes.data_as(C.c_void_p)))
            err = np.linalg.norm(y_na - y_ref) / np.linalg.norm(y_ref)
            assert err <= 1e-12, (call, err)
    finally:
        L.p3d_op_destroy(h)


def test_noalloc_rejects_meshes_above_the_limit(cuda):
    L, h, n = _op(17, seed=4)  # 3 * 35^3 = 128,625 dofs > 107,811
    try:
        x = np.zeros(n)
        y = np.zeros(n)
        rc = L.p3d_a11_apply_host_noalloc(h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p))
        assert rc == _lib.P3D_ERR_ARG
        assert b"static limit" in L.p3d_last_error()
    finally:
        L.p3d_op_destroy(h)
