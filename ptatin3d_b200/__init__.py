"""ptatin3d_b200: B200-native (sm_100a) matrix-free Q2-P1disc Stokes operators
for pTatin3d, behind a plain C ABI (include/p3d_b200.h).

The arithmetic lives in the in-tree CUDA library libp3d_b200.so; importing a
class that needs it without the library raises (there is no CPU fallback).
"""
from ._lib import (BC_MATMULT, BC_NONE, COARSE_ETA_GEOMEAN, COARSE_ETA_Q1, COARSE_GALERKIN, COARSE_REDISC,
                   GEOM_AFFINE, GEOM_AUTO, GEOM_GENERAL, PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN, SCHUR_ETA_QP, P3DError,
                   bc_bit, launch_count, lib)

__all__ = ["lib", "P3DError", "bc_bit", "launch_count", "PREC_F64", "PREC_F32", "GEOM_AUTO", "GEOM_GENERAL",
           "GEOM_AFFINE", "BC_NONE", "BC_MATMULT", "COARSE_GALERKIN", "COARSE_REDISC", "COARSE_ETA_GEOMEAN",
           "COARSE_ETA_Q1", "SCHUR_ETA_QP", "SCHUR_ETA_GEOMEAN"]
