"""Device-resident Stokes solve (FGMRES + Schur upper + GMG) from Python.

Mirrors the reference driver's linear solve
(pTatin3d_linear_viscous_forward_model_driver, src/ptatin_driver_linear_ts.c:884-1100)
for one whole mesh: build the operators on a hierarchy, set the body-force
right-hand side, solve to a relative residual tolerance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import PREC_F32, PREC_F64, SolverOpts, SolveStats, check, lib
from .operators import _check_size, _ptr, mesh_desc_whole


def default_opts(**kw) -> SolverOpts:
    o = SolverOpts()
    check(lib().p3d_solver_default_opts(C.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def max_levels(m: int, coarse_min: int = 2) -> int:
    """Levels such that the mesh halves cleanly down to a coarse size >= coarse_min."""
    lev = 1
    while m % 2 == 0 and m // 2 >= coarse_min:
        m //= 2
        lev += 1
    return lev


class StokesSolver:
    def __init__(self, mx, my, mz, dirichlet, device=0, **opts):
        self.dims = (mx, my, mz)
        self.desc = mesh_desc_whole(mx, my, mz, dirichlet)
        self.opts = default_opts(**opts)
        h = C.c_void_p()
        check(lib().p3d_solver_create(C.byref(self.desc), C.byref(self.opts), device, C.byref(h)))
        self.h = h
        self.nu = 3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1)
        self.np = 4 * mx * my * mz
        self.device = torch.device("cuda", device)

    def _dev(self, a, n=None, name="array"):
        """FP64 contiguous copy on the solver's device; n: required element count."""
        if isinstance(a, torch.Tensor):
            t = a.to(device=self.device, dtype=torch.float64).contiguous()
        else:
            t = torch.tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(-1), device=self.device)
        if n is not None:
            _check_size(t, n, torch.float64, name)
        return t

    def setup(self, coords, eta, eta_nodes=None):
        """eta_nodes: the finest level's nodal viscosity for the Q1 coefficient
        hierarchy (the reference's projection type 1), else None."""
        nel = self.dims[0] * self.dims[1] * self.dims[2]
        c, e = self._dev(coords, self.nu, "coords"), self._dev(eta, 27 * nel, "eta")
        if eta_nodes is None:
            check(lib().p3d_solver_setup(self.h, _ptr(c), _ptr(e)))
        else:
            v = self._dev(eta_nodes, self.nu // 3, "eta_nodes")
            check(lib().p3d_solver_setup_nodal(self.h, _ptr(c), _ptr(e), _ptr(v)))

    def set_rhs_body_force(self, rho, g=(0.0, 0.0, -1.0)):
        r = self._dev(rho, 27 * self.dims[0] * self.dims[1] * self.dims[2], "rho")
        check(lib().p3d_solver_set_rhs_body_force(self.h, _ptr(r), *map(float, g)))

    def set_rhs(self, bu, bp):
        bu_d, bp_d = self._dev(bu, self.nu, "bu"), self._dev(bp, self.np, "bp")  # both alive across the call
        check(lib().p3d_solver_set_rhs(self.h, _ptr(bu_d), _ptr(bp_d)))

    def solve(self, u=None, p=None, raise_on_noconv=True):
        u = torch.zeros(self.nu, dtype=torch.float64, device=self.device) if u is None else self._dev(u, self.nu, "u")
        p = torch.zeros(self.np, dtype=torch.float64, device=self.device) if p is None else self._dev(p, self.np, "p")
        st = SolveStats()
        rc = lib().p3d_solver_solve(self.h, _ptr(u), _ptr(p), C.byref(st))
        if rc != 0 and (raise_on_noconv or rc != _lib.P3D_ERR_NOCONV):
            check(rc)
        stats = {f: getattr(st, f) for f, _ in SolveStats._fields_}
        return u, p, stats

    def apply_pc(self, ru, rp):
        zu = torch.empty(self.nu, dtype=torch.float64, device=self.device)
        zp = torch.empty(self.np, dtype=torch.float64, device=self.device)
        ru_d, rp_d = self._dev(ru, self.nu, "ru"), self._dev(rp, self.np, "rp")  # both alive across the call
        check(lib().p3d_solver_apply_pc(self.h, _ptr(ru_d), _ptr(rp_d), _ptr(zu), _ptr(zp)))
        return zu, zp

    def level_apply(self, level, x):
        """FP64 velocity operator of multigrid level `level` (0 = coarsest)."""
        f = 1 << (self.opts.nlevels - 1 - int(level))
        n = 3 * (2 * (self.dims[0] // f) + 1) * (2 * (self.dims[1] // f) + 1) * (2 * (self.dims[2] // f) + 1)
        xd = self._dev(x, n, "x")
        y = torch.empty_like(xd)
        check(lib().p3d_solver_level_apply(self.h, int(level), _ptr(xd), _ptr(y)))
        return y

    def destroy(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().p3d_solver_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def solve_grouped(solvers, us=None, ps=None):
    """Solve several StokesSolver objects of one mesh shape and option set
    together (p3d_solver_solve_grouped): one launch per kernel for all of
    them, each keeping its own Krylov iteration.  Returns [(u, p, stats,
    status), ...] in the order given."""
    k = len(solvers)
    us = [None] * k if us is None else us
    ps = [None] * k if ps is None else ps
    U = [torch.zeros(S.nu, dtype=torch.float64, device=S.device) if u is None else S._dev(u, S.nu, "u")
         for S, u in zip(solvers, us)]
    P = [torch.zeros(S.np, dtype=torch.float64, device=S.device) if p is None else S._dev(p, S.np, "p")
         for S, p in zip(solvers, ps)]
    VP = C.c_void_p * k
    stats = (SolveStats * k)()
    status = (C.c_int32 * k)()
    rc = lib().p3d_solver_solve_grouped(VP(*[S.h.value for S in solvers]), k, VP(*[u.data_ptr() for u in U]),
                                        VP(*[p.data_ptr() for p in P]), C.cast(stats, C.c_void_p), status)
    if rc not in (0, _lib.P3D_ERR_NOCONV, _lib.P3D_ERR_BREAKDOWN, _lib.P3D_ERR_CANCELLED):
        check(rc)
    out = []
    for i in range(k):
        st = {f: getattr(stats[i], f) for f, _ in SolveStats._fields_}
        out.append((U[i], P[i], st, int(status[i])))
    return out
