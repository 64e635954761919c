"""The reference-side binding (ptatin3d_b200/binding/stokes_operators_b200.c),
compiled against the PETSc stand-in headers and called through the SpMVOp
function pointers of a struct _p_MatA11MF (include/stokes_operators.h:47-62)
the way MatMult_MFStokes_A11 calls a back end (src/stokes_operators.c:1185):
its result on the reference's pageable local arrays equals the reference's
own MFStokesWrapper_A11_AVX on the same inputs, and a change of the Mat's
state re-uploads the coefficients (and only then)."""
import ctypes as C
import os

import numpy as np
import pytest

from cases import rel
from ptatin3d_b200 import mesh as M

BIND = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libp3dbind.so")
_dp = C.POINTER(C.c_double)


def _binding():
    if not os.path.exists(BIND):
        pytest.skip("binding harness not built (pTatin3d sources absent when oracle/_ref was built)")
    L = C.CDLL(BIND)
    for f in ("bind_setup", "bind_touch", "bind_destroy"):
        getattr(L, f).restype = C.c_int
    L.bind_matmult.argtypes = [_dp, _dp]
    L.bind_matmult.restype = C.c_int
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


def test_binding_exports_the_spmvop_triple():
    L = _binding()
    for f in ("MFA11SetUp_B200", "MFStokesWrapper_A11_B200", "MFA11Destroy_B200"):
        assert hasattr(L, f)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,deform", [((7, 5, 6), 0.2), ((16, 16, 16), 0.0)])
def test_binding_matmult_matches_reference_avx(cuda, reference_kernels, dims, deform):
    L = _binding()
    mx, my, mz = dims
    c = M.uniform_coords(mx, my, mz)
    if deform:
        c = M.perturb_interior(c, mx, my, mz, frac=deform, seed=2)
    rng = np.random.default_rng(sum(dims))
    eta1 = 10 ** rng.uniform(-2, 2, size=(mx * my * mz, 27))
    eta2 = 10 ** rng.uniform(-2, 2, size=(mx * my * mz, 27))
    x = rng.uniform(-1, 1, size=c.size)
    y = np.zeros(c.size)  # the caller's (pageable) local arrays, kept for the back end's lifetime
    reference_kernels.setup(dims, c, eta1)
    assert L.bind_setup() == 0
    try:
        ref1 = reference_kernels.a11_raw(x, "avx")
        for _ in range(2):  # the first call uploads the coefficients, the second reuses them
            y[:] = 0.0
            assert L.bind_matmult(_p(x), _p(y)) == 0
            assert rel(y, ref1) <= 1e-12
        # new coefficients in the quadrature records: ignored until the Mat's state advances
        reference_kernels.setup(dims, c, eta2)
        y[:] = 0.0
        assert L.bind_matmult(_p(x), _p(y)) == 0
        assert rel(y, ref1) <= 1e-12
        assert L.bind_touch() == 0
        y[:] = 0.0
        assert L.bind_matmult(_p(x), _p(y)) == 0
        assert rel(y, reference_kernels.a11_raw(x, "avx")) <= 1e-12
    finally:
        assert L.bind_destroy() == 0
