"""Material points onto Gauss points: the reference's rheology-update
projections, run by libp3d_b200.so.

``update_gauss_properties`` mirrors the ``coefficient_projection_type``
switch of pTatin_EvaluateRheologyNonlinearities (src/rheology.c:150-185):

  PROJ_NULL (-1)            keep the Gauss-point values
  PROJ_P0_ARITHMETIC (0),
  PROJ_P0_HARMONIC (10),
  PROJ_P0_GEOMETRIC (20)    MPntPStokesProj_P0 (src/material_point_utils.c:2796)
  PROJ_Q1 (1)               SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes (:842)
  PROJ_ONE2ONE (4)          SwarmUpdateGaussPropertiesOne2OneMap_MPntPStokes (:803)

The markers are given as the fields of the reference's MPntStd / MPntPStokes
records that these projections read: ``wil`` (element index), ``xi`` (local
coordinates), ``eta`` and ``rho``.  The mesh is one whole mx*my*mz block.
Unknown types raise P3DError, as the reference's SETERRQ does.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import (PROJ_NULL, PROJ_ONE2ONE, PROJ_P0_ARITHMETIC, PROJ_P0_GEOMETRIC, PROJ_P0_HARMONIC, PROJ_Q1,
                   check, lib)
from .operators import _check_size, _ptr, _stream

__all__ = ["update_gauss_properties", "PROJ_NULL", "PROJ_P0_ARITHMETIC", "PROJ_P0_HARMONIC", "PROJ_P0_GEOMETRIC",
           "PROJ_Q1", "PROJ_ONE2ONE"]


def update_gauss_properties(m, projection_type, wil, xi, eta_p, rho_p, eta_q=None, rho_q=None, nodal=False):
    """Gauss-point viscosity and density [nel, 27] of the mesh m = (mx, my, mz)
    from n markers: wil int32 [n], xi float64 [n, 3], eta_p / rho_p float64 [n]
    (CUDA tensors).  eta_q / rho_q are updated in place when given (PROJ_NULL
    leaves them unchanged), else allocated.  nodal=True (PROJ_Q1) also returns
    the nodal viscosity on the Q2 lattice, the input of the solver's Q1
    coefficient hierarchy (StokesSolver.setup(..., eta_nodes=...))."""
    mx, my, mz = m
    nel = mx * my * mz
    dev = eta_p.device
    if eta_q is None:
        eta_q = torch.zeros(nel, 27, dtype=torch.float64, device=dev)
    if rho_q is None:
        rho_q = torch.zeros(nel, 27, dtype=torch.float64, device=dev)
    n = wil.numel()
    nb = C.c_int64()
    check(lib().p3d_marker_project_workspace(mx, my, mz, projection_type, C.byref(nb)))
    ws = torch.empty(max(1, nb.value // 8), dtype=torch.float64, device=dev)
    xc = xi.contiguous() if xi is not None else None  # kept alive until the launch is queued
    for t, k, dt, name in ((wil, n, torch.int32, "wil"), (xc, 3 * n, torch.float64, "xi"),
                           (eta_p, n, torch.float64, "eta_p"), (rho_p, n, torch.float64, "rho_p"),
                           (eta_q, 27 * nel, torch.float64, "eta_q"), (rho_q, 27 * nel, torch.float64, "rho_q")):
        if t is not None:
            _check_size(t, k, dt, name)
    check(lib().p3d_marker_project(mx, my, mz, projection_type, n, _ptr(wil), None if xc is None else _ptr(xc),
                                   _ptr(eta_p), _ptr(rho_p), _ptr(eta_q), _ptr(rho_q), _ptr(ws), _stream()))
    if nodal:
        if projection_type != PROJ_Q1:
            raise ValueError("the nodal field exists for the Q1 projection only")
        nn = (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1)
        return eta_q, rho_q, ws[:nn]
    return eta_q, rho_q
