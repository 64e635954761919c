"""The C-ABI library loads and exports every entry point include/*.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes as C
import glob
import os
import re
import subprocess

from ptatin3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(p3d_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in sorted(declared()) if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (p3d_\w+)", out))
    assert declared() <= exported, declared() - exported


def test_bindings_cover_header():
    assert declared() <= set(_lib.exported_symbols())


def test_errors_are_codes_not_exits():
    L = _lib.lib()
    d = _lib.MeshDesc()
    assert L.p3d_mesh_desc_whole(0, 1, 1, 0, C.byref(d)) == _lib.P3D_ERR_ARG
    assert b"bad sizes" in L.p3d_last_error()
    assert L.p3d_op_create(None, 64, 0, None) == _lib.P3D_ERR_ARG
    assert L.p3d_a11_apply(None, None, None, None) == _lib.P3D_ERR_ARG
    assert L.p3d_mg_prolong(16, 2, 2, 2, 3, None, None, None) == _lib.P3D_ERR_ARG


def test_inconsistent_ghosted_desc_is_refused():
    """Host-side validation of a ghosted local-array descriptor, before any device call."""
    L = _lib.lib()
    d = _lib.MeshDesc()
    assert L.p3d_mesh_desc_whole(4, 3, 5, 0, C.byref(d)) == 0
    h = C.c_void_p()
    d.ox = 2  # 2 + 2*4 + 1 > gx = 9
    assert L.p3d_op_create(C.byref(d), 64, 0, C.byref(h)) == _lib.P3D_ERR_ARG
    assert b"exceeds the ghosted lattice" in L.p3d_last_error()
    d.ox, d.oy = 0, -1
    assert L.p3d_op_create(C.byref(d), 64, 0, C.byref(h)) == _lib.P3D_ERR_ARG
    d.oy = 0
    assert L.p3d_op_create(C.byref(d), 16, 0, C.byref(h)) == _lib.P3D_ERR_ARG
    assert b"precision" in L.p3d_last_error()


def test_mesh_desc_whole():
    d = _lib.MeshDesc()
    assert _lib.lib().p3d_mesh_desc_whole(4, 5, 6, 7, C.byref(d)) == 0
    assert (d.gx, d.gy, d.gz, d.ox, d.global_faces) == (9, 11, 13, 0, 0x3F)


def test_solver_options_defaults_and_checks():
    """Option defaults and validation happen on the host, before any device call."""
    L = _lib.lib()
    o = _lib.SolverOpts()
    assert L.p3d_solver_default_opts(C.byref(o)) == 0
    assert (o.nlevels, o.cheb_its, o.restart, o.inner_its, o.coarse_op, o.schur_eta) == \
        (4, 3, 30, 0, _lib.COARSE_GALERKIN, _lib.SCHUR_ETA_QP)
    assert (o.cheb_lo, o.cheb_hi) == (0.2, 1.1)
    d = _lib.MeshDesc()
    assert L.p3d_mesh_desc_whole(16, 16, 16, 0, C.byref(d)) == 0
    h = C.c_void_p()
    o.restart = _lib.MAX_RESTART + 1
    assert L.p3d_solver_create(C.byref(d), C.byref(o), 0, C.byref(h)) == _lib.P3D_ERR_ARG
    o.restart = 30
    o.nlevels = 1  # 16^3 coarse level: 107,811 dofs, above the dense limit
    assert L.p3d_solver_create(C.byref(d), C.byref(o), 0, C.byref(h)) == _lib.P3D_ERR_ARG
    assert b"dense limit" in L.p3d_last_error()
    o.nlevels, o.schur_eta = 3, 7
    assert L.p3d_solver_create(C.byref(d), C.byref(o), 0, C.byref(h)) == _lib.P3D_ERR_ARG


def test_marker_projection_arguments_checked_on_host():
    """Workspace sizes and argument errors of p3d_marker_project need no device."""
    L = _lib.lib()
    nb = C.c_int64()
    assert L.p3d_marker_project_workspace(3, 2, 4, _lib.PROJ_Q1, C.byref(nb)) == 0
    assert nb.value == 3 * 7 * 5 * 9 * 8  # three node-lattice fields
    assert L.p3d_marker_project_workspace(3, 2, 4, _lib.PROJ_P0_GEOMETRIC, C.byref(nb)) == 0
    assert nb.value == 3 * 24 * 8  # three sums per element
    assert L.p3d_marker_project_workspace(3, 2, 4, _lib.PROJ_ONE2ONE, C.byref(nb)) == 0 and nb.value == 0
    assert L.p3d_marker_project_workspace(3, 2, 4, 2, C.byref(nb)) == _lib.P3D_ERR_ARG  # Q2: not supported
    assert L.p3d_marker_project(3, 2, 4, _lib.PROJ_NULL, 0, *([None] * 8)) == 0
    assert L.p3d_marker_project(3, 2, 4, 3, 0, *([None] * 8)) == _lib.P3D_ERR_ARG
    assert b"unknown projection type" in L.p3d_last_error()
    buf = (C.c_double * 4)()
    ptr = C.cast(buf, C.c_void_p)
    assert L.p3d_marker_project(3, 2, 4, _lib.PROJ_ONE2ONE, 5, ptr, None, ptr, ptr, ptr, ptr, None, None) \
        == _lib.P3D_ERR_ARG
    assert b"27 markers per element" in L.p3d_last_error()
    assert L.p3d_marker_project(3, 2, 4, _lib.PROJ_Q1, 5, ptr, None, ptr, ptr, ptr, ptr, ptr, None) \
        == _lib.P3D_ERR_ARG  # Q1 needs xi


def test_python_wrappers_refuse_wrong_sizes():
    """The torch-facing wrappers check every buffer's element count and type
    before a pointer reaches the library, so a wrong size is an error on the
    host and never an out-of-bounds access on the device."""
    import pytest
    import torch

    from ptatin3d_b200.markers import PROJ_Q1, update_gauss_properties
    from ptatin3d_b200.operators import mg_prolong
    wil = torch.zeros(5, dtype=torch.int32)
    one = torch.ones(5, dtype=torch.float64)
    with pytest.raises(_lib.P3DError, match="xi"):
        update_gauss_properties((2, 2, 2), PROJ_Q1, wil, torch.zeros(4, 3, dtype=torch.float64), one, one)
    with pytest.raises(_lib.P3DError, match="eta_q"):
        update_gauss_properties((2, 2, 2), PROJ_Q1, wil, torch.zeros(5, 3, dtype=torch.float64), one, one,
                                torch.zeros(7, 27, dtype=torch.float64), torch.zeros(8, 27, dtype=torch.float64))
    with pytest.raises(_lib.P3DError, match="wil"):
        update_gauss_properties((2, 2, 2), PROJ_Q1, wil.long(), torch.zeros(5, 3, dtype=torch.float64), one, one)
    with pytest.raises(_lib.P3DError, match="xf"):
        mg_prolong(torch.zeros(3 * 8, dtype=torch.float64), torch.zeros(3 * 26, dtype=torch.float64), (2, 2, 2))


def test_c_caller_links_and_runs(tmp_path):
    """The header compiles as C99 and a C program links libp3d_b200.so and
    calls it with plain pointers (the entry points that need no device)."""
    import shutil

    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = str(tmp_path / "capi_host")
    _lib.lib()  # the CUDA runtime this process resolved for the library
    maps = open("/proc/self/maps").read().split()
    cuda_rt = next((os.path.dirname(f) for f in maps if "libcudart.so" in f), None)
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "capi_host.c"), "-L", libdir, "-lp3d_b200", f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ)
    if cuda_rt:
        env["LD_LIBRARY_PATH"] = cuda_rt + ":" + env.get("LD_LIBRARY_PATH", "")
    out = subprocess.run([exe], capture_output=True, text=True, env=env)
    assert out.returncode == 0, out.stderr
    lines = dict(l.split(" ", 1) for l in out.stdout.strip().splitlines())
    assert lines["desc"] == "0 4 9 7 11 0 0 1 63"
    assert lines["bad_desc"] == f"{_lib.P3D_ERR_ARG} msg"
    assert lines["ws_q1"] == f"0 {3 * 9 * 7 * 11 * 8}"
    assert lines["ws_p0"] == f"0 {3 * 60 * 8}"
    assert lines["solver"] == "0 4 0 1"
    assert lines["version"].startswith("p3d_b200")
