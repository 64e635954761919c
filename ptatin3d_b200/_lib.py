"""ctypes binding of the in-tree CUDA library ``libp3d_b200.so``.

The library is the product: there is no CPU fallback.  Loading fails loudly
when the shared object is missing, and every call that reports a nonzero
status raises :class:`P3DError` with the library's message (the C ABI never
exits the process, unlike the reference CUDA backend's CUDACHECK at
src/stokes_operators_cuda.cu:46-57).
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libp3d_b200.so")

P3D_OK = 0
(P3D_ERR_ARG, P3D_ERR_CUDA, P3D_ERR_STATE, P3D_ERR_NOMEM, P3D_ERR_NOCONV, P3D_ERR_BREAKDOWN, P3D_ERR_TIMEOUT,
 P3D_ERR_CANCELLED) = range(1, 9)
PREC_F64, PREC_F32 = 64, 32
COARSE_GALERKIN, COARSE_REDISC = 0, 1
SCHUR_ETA_QP, SCHUR_ETA_GEOMEAN = 0, 1
COARSE_ETA_GEOMEAN, COARSE_ETA_Q1 = 0, 1
MAX_RESTART = 120
COARSE_MAX_DOFS = 16384
NOALLOC_MAX_DOFS = 107811  # P3D_NOALLOC_MAX_DOFS
GEOM_AUTO, GEOM_GENERAL, GEOM_AFFINE = 0, 1, 2
BC_NONE, BC_MATMULT = 0, 1
PROJ_NULL, PROJ_P0_ARITHMETIC, PROJ_Q1, PROJ_ONE2ONE, PROJ_P0_HARMONIC, PROJ_P0_GEOMETRIC = -1, 0, 1, 4, 10, 20
FACE_IMIN, FACE_IMAX, FACE_JMIN, FACE_JMAX, FACE_KMIN, FACE_KMAX = range(6)


def bc_bit(face: int, comp: int) -> int:
    return 1 << (3 * face + comp)


class P3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"p3d error {code}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("mx", C.c_int32), ("my", C.c_int32), ("mz", C.c_int32),
                ("gx", C.c_int32), ("gy", C.c_int32), ("gz", C.c_int32),
                ("ox", C.c_int32), ("oy", C.c_int32), ("oz", C.c_int32),
                ("dirichlet", C.c_uint32), ("global_faces", C.c_uint32)]


class SolverOpts(C.Structure):
    _fields_ = [("nlevels", C.c_int32), ("cheb_its", C.c_int32), ("cheb_lo", C.c_double), ("cheb_hi", C.c_double),
                ("esteig_its", C.c_int32), ("mg_precision", C.c_int32), ("restart", C.c_int32),
                ("max_it", C.c_int32), ("rtol", C.c_double), ("atol", C.c_double), ("use_graph", C.c_int32),
                ("verbose", C.c_int32), ("inner_its", C.c_int32), ("coarse_op", C.c_int32),
                ("schur_eta", C.c_int32), ("coarse_eta", C.c_int32), ("inner_rtol", C.c_double)]


class Request(C.Structure):
    _fields_ = [("mx", C.c_int32), ("my", C.c_int32), ("mz", C.c_int32), ("dirichlet", C.c_uint32),
                ("coords", C.c_void_p), ("eta", C.c_void_p), ("rho", C.c_void_p),
                ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
                ("u", C.c_void_p), ("p", C.c_void_p), ("opts", SolverOpts), ("tag", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("tag", C.c_int64), ("status", C.c_int32), ("iterations", C.c_int32), ("rel_residual", C.c_double),
                ("wait_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64), ("active", C.c_int32),
                ("queued", C.c_int32), ("device_bytes", C.c_int64), ("peak_device_bytes", C.c_int64),
                ("solvers_created", C.c_int32), ("solvers_reused", C.c_int32), ("grouped", C.c_int64),
                ("groups", C.c_int64)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("r0", C.c_double), ("rfinal", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double), ("lmax_fine", C.c_double),
                ("coarse_dofs", C.c_int32), ("inner_iterations", C.c_int32), ("group_members", C.c_int32)]


_lib = None

_SIGS = {
    "p3d_solver_default_opts": ([C.POINTER(SolverOpts)], C.c_int),
    "p3d_solver_create": ([C.POINTER(MeshDesc), C.POINTER(SolverOpts), C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "p3d_solver_setup": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_solver_setup_nodal": ([C.c_void_p] * 4, C.c_int),
    "p3d_solver_set_rhs_body_force": ([C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "p3d_solver_set_rhs": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_solver_solve": ([C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveStats)], C.c_int),
    "p3d_solver_apply_pc": ([C.c_void_p] * 5, C.c_int),
    "p3d_solver_destroy": ([C.c_void_p], C.c_int),
    "p3d_solver_level_apply": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_solver_estimate_bytes": ([C.POINTER(MeshDesc), C.POINTER(SolverOpts), C.POINTER(C.c_int64)], C.c_int),
    "p3d_server_create": ([C.c_int, C.c_int64, C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "p3d_server_submit": ([C.c_void_p, C.POINTER(Request)], C.c_int),
    "p3d_server_poll": ([C.c_void_p, C.POINTER(Result), C.c_int32, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "p3d_server_get_stats": ([C.c_void_p, C.POINTER(ServerStats)], C.c_int),
    "p3d_server_destroy": ([C.c_void_p], C.c_int),
    "p3d_last_error": ([], C.c_char_p),
    "p3d_kernel_launch_count": ([], C.c_int64),
    "p3d_version": ([], C.c_char_p),
    "p3d_mesh_desc_whole": ([C.c_int32, C.c_int32, C.c_int32, C.c_uint32, C.POINTER(MeshDesc)], C.c_int),
    "p3d_op_create": ([C.POINTER(MeshDesc), C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "p3d_op_destroy": ([C.c_void_p], C.c_int),
    "p3d_op_set_coefficients": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "p3d_op_set_coefficients_device": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "p3d_op_set_bc_mode": ([C.c_void_p, C.c_int], C.c_int),
    "p3d_op_geometry_mode": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "p3d_op_sizes": ([C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "p3d_a11_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_op_set_host_chunks": ([C.c_void_p, C.c_int], C.c_int),
    "p3d_stokes_residual": ([C.c_void_p] * 9, C.c_int),
    "p3d_a11_mult": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_a11_diagonal": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_a12_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_a21_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_stokes_apply": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_a11_apply_host": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_a11_apply_host_noalloc": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_op_set_host_register": ([C.c_void_p, C.c_int], C.c_int),
    "p3d_server_cancel": ([C.c_void_p, C.c_int64], C.c_int),
    "p3d_server_set_group_max": ([C.c_void_p, C.c_int32], C.c_int),
    "p3d_server_set_group_elements": ([C.c_void_p, C.c_int64], C.c_int),
    "p3d_server_set_group_overtake_ms": ([C.c_void_p, C.c_int32], C.c_int),
    "p3d_solver_solve_grouped": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                  C.c_void_p, C.POINTER(C.c_int32)], C.c_int),
    "p3d_a11_mult_grouped": ([C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32,
                              C.c_void_p], C.c_int),
    "p3d_slab_add_plane": ([C.c_int, C.c_int32, C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p], C.c_int),
    "p3d_debug_fail_allocations_after": ([C.c_int64], C.c_int),
    "p3d_debug_poison_allocations": ([C.c_int32], C.c_int),
    "p3d_mg_prolong": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_mg_restrict": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "p3d_marker_project_workspace": ([C.c_int32, C.c_int32, C.c_int32, C.c_int, C.POINTER(C.c_int64)], C.c_int),
    "p3d_marker_project": ([C.c_int32, C.c_int32, C.c_int32, C.c_int, C.c_int64] + [C.c_void_p] * 8, C.c_int),
}


def lib():
    """Load libp3d_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ptatin3d_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def exported_symbols():
    return list(_SIGS)


def check(rc: int):
    if rc != P3D_OK:
        raise P3DError(rc, lib().p3d_last_error().decode())


def launch_count() -> int:
    return int(lib().p3d_kernel_launch_count())
