"""Host-side mirror of pTatin3d's matrix-free Stokes operator interface.

The classes keep the reference's names and contracts so code written against
the reference reads the same way:

  MatA11MF   <-> struct _p_MatA11MF + MatMult_MFStokes_A11 /
                 MatGetDiagonal_MFStokes_A11 (src/stokes_operators.c:101-334,
                 1060-1205); ``spmv`` is the SpMVOp_MatMult callback contract
                 (include/stokes_operators.h:59-61): y += sum_e A_e x on the
                 ghosted local arrays, no boundary handling.
  MatStokesMF<-> struct _p_MatStokesMF + MatMult_MFStokes_A12/_A21/_A
                 (src/stokes_operators.c:884-967, 1284-1486).

All arrays are torch CUDA tensors (device memory and streams only; the
arithmetic runs in libp3d_b200.so).  Errors raise P3DError, mirroring the
reference's PetscErrorCode returns.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import BC_MATMULT, BC_NONE, GEOM_AUTO, PREC_F32, PREC_F64, MeshDesc, check, lib


def _ptr(t: torch.Tensor):
    if not t.is_cuda:
        raise _lib.P3DError(_lib.P3D_ERR_ARG, "expected a CUDA tensor")
    if not t.is_contiguous():
        raise _lib.P3DError(_lib.P3D_ERR_ARG, "expected a contiguous tensor")
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_size(t: torch.Tensor, n: int, dtype, name: str):
    """Raise unless t holds exactly n elements of dtype (the library reads or
    writes n elements through its pointer)."""
    if t.dtype != dtype or t.numel() != n:
        raise _lib.P3DError(_lib.P3D_ERR_ARG, f"{name}: expected {n} x {dtype}, got {t.numel()} x {t.dtype}")


def _sized(t: torch.Tensor, n: int, dtype, name: str):
    """Pointer of a contiguous CUDA tensor of exactly n elements of dtype."""
    _check_size(t, n, dtype, name)
    return _ptr(t)


def mesh_desc_whole(mx, my, mz, dirichlet=0) -> MeshDesc:
    d = MeshDesc()
    check(lib().p3d_mesh_desc_whole(mx, my, mz, dirichlet, C.byref(d)))
    return d


class _Op:
    """One p3d_op handle: mesh + coefficients resident in HBM."""

    def __init__(self, desc: MeshDesc, precision=PREC_F64, device=0):
        self.desc = desc
        self.precision = precision
        self.dtype = torch.float64 if precision == PREC_F64 else torch.float32
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        check(lib().p3d_op_create(C.byref(desc), precision, device, C.byref(h)))
        self.h = h
        nv, np_ = C.c_int64(), C.c_int64()
        check(lib().p3d_op_sizes(h, C.byref(nv), C.byref(np_)))
        self.n_velocity, self.n_pressure = nv.value, np_.value

    def set_coefficients(self, coords, eta, geom=GEOM_AUTO):
        """coords: (3*gx*gy*gz,) float64, eta: (nel*27,) float64 -- host numpy or CUDA tensors."""
        nc = 3 * self.desc.gx * self.desc.gy * self.desc.gz
        ne = 27 * self.desc.mx * self.desc.my * self.desc.mz
        if isinstance(coords, torch.Tensor) and coords.is_cuda:
            c = coords.to(torch.float64).contiguous()
            e = eta.to(device=c.device, dtype=torch.float64).contiguous()
            check(lib().p3d_op_set_coefficients_device(self.h, _sized(c, nc, torch.float64, "coords"),
                                                       _sized(e, ne, torch.float64, "eta"), geom))
        else:
            c = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1)
            e = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
            if c.size != nc:
                raise _lib.P3DError(_lib.P3D_ERR_ARG, f"coords has {c.size} entries")
            if e.size != ne:
                raise _lib.P3DError(_lib.P3D_ERR_ARG, f"eta has {e.size} entries")
            check(lib().p3d_op_set_coefficients(self.h, c.ctypes.data_as(C.c_void_p),
                                                e.ctypes.data_as(C.c_void_p), geom))

    @property
    def geometry_mode(self) -> int:
        m = C.c_int()
        check(lib().p3d_op_geometry_mode(self.h, C.byref(m)))
        return m.value

    def _bc(self, mode):
        check(lib().p3d_op_set_bc_mode(self.h, mode))

    def _vec(self, t, n, name):
        return _sized(t, n, self.dtype, name)

    def destroy(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().p3d_op_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class MatA11MF(_Op):
    """Matrix-free viscous block A11 of one mesh (MatA11MFCreate + MatA11MFSetup)."""

    def spmv(self, x_loc: torch.Tensor, y_loc: torch.Tensor):
        """SpMVOp_MatMult contract: y_loc += sum_e A_e x_loc (caller handles BCs)."""
        self._bc(BC_NONE)
        check(lib().p3d_a11_apply(self.h, self._vec(x_loc, self.n_velocity, "x"),
                                  self._vec(y_loc, self.n_velocity, "y"), _stream()))

    def mult(self, x: torch.Tensor, y: torch.Tensor):
        """MatMult_MFStokes_A11: y = A11 x with Dirichlet columns zeroed and rows y_k = x_k."""
        self._bc(BC_MATMULT)
        check(lib().p3d_a11_mult(self.h, self._vec(x, self.n_velocity, "x"),
                                 self._vec(y, self.n_velocity, "y"), _stream()))

    def mult_add(self, x: torch.Tensor, y: torch.Tensor):
        """y += A11 x with the MatMult boundary convention (Dirichlet rows overwritten)."""
        self._bc(BC_MATMULT)
        check(lib().p3d_a11_apply(self.h, self._vec(x, self.n_velocity, "x"),
                                  self._vec(y, self.n_velocity, "y"), _stream()))

    def get_diagonal(self, d: torch.Tensor, boundary=True):
        """MatGetDiagonal_MFStokes_A11: d = diag(A11), Dirichlet slots = 1."""
        d.zero_()
        self._bc(BC_MATMULT if boundary else BC_NONE)
        check(lib().p3d_a11_diagonal(self.h, self._vec(d, self.n_velocity, "d"), _stream()))

    def mult_host(self, x: np.ndarray, y: np.ndarray, boundary=False):
        """Host-buffer apply (reference CUDA backend contract): y = A11 x, synchronous."""
        self._bc(BC_MATMULT if boundary else BC_NONE)
        x = np.ascontiguousarray(x, dtype=np.float64)
        if not (y.flags.c_contiguous and y.dtype == np.float64):
            raise _lib.P3DError(_lib.P3D_ERR_ARG, "y must be a contiguous float64 array")
        check(lib().p3d_a11_apply_host(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p)))


class MatStokesMF(MatA11MF):
    """Full Stokes operator blocks [A11 A12; A21 0] on one mesh (MatStokesMF)."""

    def mult_a12(self, p: torch.Tensor, yu: torch.Tensor, boundary=True):
        """MatMult_MFStokes_A12: yu = A12 p, Dirichlet rows zeroed."""
        yu.zero_()
        self._bc(BC_MATMULT if boundary else BC_NONE)
        check(lib().p3d_a12_apply(self.h, self._vec(p, self.n_pressure, "p"),
                                  self._vec(yu, self.n_velocity, "yu"), _stream()))

    def mult_a21(self, u: torch.Tensor, yp: torch.Tensor, boundary=True):
        """MatMult_MFStokes_A21: yp = A21 u with Dirichlet columns of u zeroed."""
        yp.zero_()
        self._bc(BC_MATMULT if boundary else BC_NONE)
        check(lib().p3d_a21_apply(self.h, self._vec(u, self.n_velocity, "u"),
                                  self._vec(yp, self.n_pressure, "yp"), _stream()))

    def mult_stokes(self, u, p, yu, yp, boundary=True):
        """MatMult_MFStokes_A: [yu; yp] = [A11 A12; A21 0][u; p]."""
        yu.zero_()
        yp.zero_()
        self._bc(BC_MATMULT if boundary else BC_NONE)
        check(lib().p3d_stokes_apply(self.h, self._vec(u, self.n_velocity, "u"), self._vec(p, self.n_pressure, "p"),
                                     self._vec(yu, self.n_velocity, "yu"), self._vec(yp, self.n_pressure, "yp"),
                                     _stream()))


    def residual(self, u, p, fu=None, fp=None, phi=None):
        """FormFunction_Stokes: (ru, rp) = ([A11 u + A12 p - f_u; A21 u - f_p] with the
        Dirichlet values phi inserted in u, Dirichlet rows u_k - phi_k).  fu: (nel, 27, 3)
        Gauss-point force, fp: (nel, 27), phi: Dirichlet values -- CUDA tensors or arrays."""
        def dev(a):
            if a is None:
                return None
            if isinstance(a, torch.Tensor):
                return a.to(device=self.device, dtype=torch.float64).contiguous().reshape(-1)
            return torch.tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(-1), device=self.device)
        u_d, p_d, fu_d, fp_d, phi_d = dev(u), dev(p), dev(fu), dev(fp), dev(phi)
        ru = torch.empty(self.n_velocity, dtype=torch.float64, device=self.device)
        rp = torch.empty(self.n_pressure, dtype=torch.float64, device=self.device)
        nel = self.desc.mx * self.desc.my * self.desc.mz
        opt = lambda t, n, name: None if t is None else _sized(t, n, torch.float64, name)
        check(lib().p3d_stokes_residual(self.h, self._vec(u_d, self.n_velocity, "u"), self._vec(p_d, self.n_pressure, "p"),
                                        opt(phi_d, self.n_velocity, "phi"), opt(fu_d, 81 * nel, "fu"),
                                        opt(fp_d, 27 * nel, "fp"), _ptr(ru), _ptr(rp), _stream()))
        return ru, rp


def _transfer_sizes(cn, ndof):
    nc = ndof * cn[0] * cn[1] * cn[2]
    nf = ndof * (2 * cn[0] - 1) * (2 * cn[1] - 1) * (2 * cn[2] - 1)
    return nc, nf


def mg_prolong(xc: torch.Tensor, xf: torch.Tensor, cn, ndof=3):
    """xf = P xc on the node lattice, cn coarse nodes per direction."""
    prec = PREC_F64 if xc.dtype == torch.float64 else PREC_F32
    nc, nf = _transfer_sizes(cn, ndof)
    _check_size(xf, nf, xc.dtype, "xf")
    check(lib().p3d_mg_prolong(prec, cn[0], cn[1], cn[2], ndof, _sized(xc, nc, xc.dtype, "xc"),
                               _sized(xf, nf, xc.dtype, "xf"), _stream()))


def mg_restrict(xf: torch.Tensor, xc: torch.Tensor, cn, ndof=3):
    """xc = P^T xf on the node lattice, cn coarse nodes per direction."""
    prec = PREC_F64 if xf.dtype == torch.float64 else PREC_F32
    nc, nf = _transfer_sizes(cn, ndof)
    _check_size(xc, nc, xf.dtype, "xc")
    check(lib().p3d_mg_restrict(prec, cn[0], cn[1], cn[2], ndof, _sized(xf, nf, xf.dtype, "xf"),
                                _sized(xc, nc, xf.dtype, "xc"), _stream()))
