"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two independent checkers, both plain CPU code:
  * ``Restatement`` -- oracle/liboracle.so, the C restatement in q2_oracle.c
    (and ``marker_project``, a numpy restatement of the material-point
    projections);
  * ``Reference``   -- oracle/_ref/libp3dref.so, the reference's own element
    kernels (stokes_operators_{tensor,avx,mf}.c, element_utils_q2.c),
    material-point projections (material_point_utils.c, quadrature.c), error
    norms (inorms.c) and SolCx analytic solution
    (models/analytics_vv/SolCxSolution.c), compiled unmodified against
    oracle/shim by ``make -C oracle ref``.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.  The product (ptatin3d_b200) never imports it.

MatMult conventions applied here follow src/stokes_operators.c:1142-1205
(A11), :1284-1350 (A12), :1424-1486 (A21), :1060-1099 (diagonal).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libp3dref.so")

_dp = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)


def build(ref_dir: str | None = None, quiet: bool = True) -> None:
    """Compile liboracle.so, and oracle/_ref from the pTatin3d source tree at
    ref_dir (or $P3D_REFERENCE_DIR).  Without either, only the restatement is
    built; a ref_dir that holds no src/ directory is an error."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=out)
    ref_dir = ref_dir or os.environ.get("P3D_REFERENCE_DIR")
    if not ref_dir:
        return
    if not os.path.isdir(os.path.join(ref_dir, "src")):
        raise FileNotFoundError(f"pTatin3d source tree not found: {ref_dir}/src")
    subprocess.run(["make", "-C", HERE, "ref", f"REF_DIR={ref_dir}"], check=True, stdout=out)
    if os.path.exists(os.path.join(os.path.dirname(HERE), "ptatin3d_b200", "libp3d_b200.so")):
        subprocess.run(["make", "-C", HERE, "bind", f"REF_DIR={ref_dir}"], check=True, stdout=out)


def _p(a):
    return a.ctypes.data_as(_dp)


class Restatement:
    def __init__(self):
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.o_a11_apply.argtypes = [C.c_int] * 3 + [_dp] * 4
        L.o_a21_apply.argtypes = [C.c_int] * 3 + [_dp] * 3
        L.o_a11_diag.argtypes = [C.c_int] * 3 + [_dp] * 3
        L.o_a12_apply.argtypes = [C.c_int] * 3 + [_dp] * 3
        L.o_schur_mass.argtypes = [C.c_int] * 3 + [_dp] * 3
        L.o_a11_element_matrix.argtypes = [_dp] * 3
        L.o_prolong.argtypes = [C.c_int] * 4 + [_dp] * 2
        L.o_restrict.argtypes = [C.c_int] * 4 + [_dp] * 2
        self.L = L

    # raw element operators (y += ...), SpMVOp contract
    def a11_raw(self, dims, coords, eta, x):
        y = np.zeros_like(x)
        self.L.o_a11_apply(*dims, _p(coords), _p(eta), _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y))
        return y

    def diag_raw(self, dims, coords, eta):
        nn = coords.size
        y = np.zeros(nn)
        self.L.o_a11_diag(*dims, _p(coords), _p(eta), _p(y))
        return y

    def a12_raw(self, dims, coords, p):
        y = np.zeros(coords.size)
        self.L.o_a12_apply(*dims, _p(coords), _p(np.ascontiguousarray(p, dtype=np.float64)), _p(y))
        return y

    def a21_raw(self, dims, coords, u):
        nel = dims[0] * dims[1] * dims[2]
        y = np.zeros(4 * nel)
        self.L.o_a21_apply(*dims, _p(coords), _p(np.ascontiguousarray(u, dtype=np.float64)), _p(y))
        return y

    def schur_mass(self, dims, coords, eta):
        nel = dims[0] * dims[1] * dims[2]
        S = np.zeros(16 * nel)
        self.L.o_schur_mass(*dims, _p(coords), _p(eta), _p(S))
        return S.reshape(nel, 4, 4)

    def element_matrix(self, elcoords, eta_e):
        K = np.zeros(81 * 81)
        self.L.o_a11_element_matrix(_p(np.ascontiguousarray(elcoords, dtype=np.float64)), _p(np.ascontiguousarray(eta_e, dtype=np.float64)), _p(K))
        return K.reshape(81, 81)

    def eta_hierarchy(self, dims, eta, nlevels):
        """Gauss-point viscosity of every level, finest first, by the reference's
        Q1 projection hierarchy (src/material_point_utils.c:1267-1420)."""
        for f, n in (("o_eta_project_nodes", 4), ("o_eta_restrict_nodes", 5), ("o_eta_nodes_to_qp", 5)):
            getattr(self.L, f).argtypes = [C.c_int] * 3 + [_dp] * 2
        mx, my, mz = dims
        v = np.zeros((2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
        self.L.o_eta_project_nodes(mx, my, mz, _p(np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)), _p(v))
        out = [np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)]
        for _ in range(nlevels - 1):
            mx, my, mz = mx // 2, my // 2, mz // 2
            vc = np.zeros((2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
            self.L.o_eta_restrict_nodes(2 * mx + 1, 2 * my + 1, 2 * mz + 1, _p(v), _p(vc))
            e = np.zeros(27 * mx * my * mz)
            self.L.o_eta_nodes_to_qp(mx, my, mz, _p(vc), _p(e))
            out.append(e)
            v = vc
        return out

    def eta_hierarchy_from_nodes(self, dims, eta, v, nlevels):
        """The same hierarchy started from a given finest-level nodal field v
        (the reference's projection type 1: v is the markers' Q1 nodal field,
        src/material_point_utils.c:1267-1360)."""
        for f in ("o_eta_restrict_nodes", "o_eta_nodes_to_qp"):
            getattr(self.L, f).argtypes = [C.c_int] * 3 + [_dp] * 2
        mx, my, mz = dims
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = [np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)]
        for _ in range(nlevels - 1):
            mx, my, mz = mx // 2, my // 2, mz // 2
            vc = np.zeros((2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
            self.L.o_eta_restrict_nodes(2 * mx + 1, 2 * my + 1, 2 * mz + 1, _p(v), _p(vc))
            e = np.zeros(27 * mx * my * mz)
            self.L.o_eta_nodes_to_qp(mx, my, mz, _p(vc), _p(e))
            out.append(e)
            v = vc
        return out

    def prolong(self, cn, ndof, xc):
        fn = [2 * c - 1 for c in cn]
        xf = np.zeros(fn[0] * fn[1] * fn[2] * ndof)
        self.L.o_prolong(*cn, ndof, _p(np.ascontiguousarray(xc, dtype=np.float64)), _p(xf))
        return xf

    def restrict(self, cn, ndof, xf):
        xc = np.zeros(cn[0] * cn[1] * cn[2] * ndof)
        self.L.o_restrict(*cn, ndof, _p(np.ascontiguousarray(xf, dtype=np.float64)), _p(xc))
        return xc


class Reference:
    """The reference's own kernels; one mesh at a time (module-global state in the driver)."""

    VARIANTS = {"tensor": 0, "avx": 1, "ref": 2, "loworder": 3}

    def __init__(self):
        if not os.path.exists(REF_LIB):
            build()
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError("oracle/_ref/libp3dref.so not built (pTatin3d sources absent)")
        L = C.CDLL(REF_LIB)
        L.ref_setup.argtypes = [C.c_int] * 3 + [_dp] * 2
        L.ref_a11.argtypes = [C.c_int, _dp, _dp]
        L.ref_diag.argtypes = [_dp]
        L.ref_a12.argtypes = [_dp, _dp]
        L.ref_a21.argtypes = [_dp, _dp]
        L.ref_a12_avx.argtypes = [_dp, _dp]
        L.ref_a_avx.argtypes = [_dp] * 4
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_marker_project.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int32), _dp, _dp, _dp, _dp, _dp]
        L.ref_solcx_norms.argtypes = [C.c_double] * 3 + [C.c_int] + [_dp] * 3
        L.ref_solcx_exact.argtypes = [C.c_double] * 3 + [C.c_int] + [_dp] * 3
        self.L = L
        self.dims = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_LIB)

    def setup(self, dims, coords, eta):
        self.dims = tuple(dims)
        self._coords = np.ascontiguousarray(coords, dtype=np.float64)
        self._eta = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
        rc = self.L.ref_setup(*self.dims, _p(self._coords), _p(self._eta))
        assert rc == 0

    def set_threads(self, n):
        self.L.ref_set_threads(int(n))

    def a11_raw(self, x, variant="tensor", out=None):
        y = np.zeros_like(x) if out is None else out
        rc = self.L.ref_a11(self.VARIANTS[variant], _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y))
        assert rc == 0
        return y

    def diag_raw(self):
        y = np.zeros(self._coords.size)
        assert self.L.ref_diag(_p(y)) == 0
        return y

    def a12_raw(self, p):
        y = np.zeros(self._coords.size)
        assert self.L.ref_a12(_p(np.ascontiguousarray(p, dtype=np.float64)), _p(y)) == 0
        return y

    def a21_raw(self, u):
        y = np.zeros(4 * self.dims[0] * self.dims[1] * self.dims[2])
        assert self.L.ref_a21(_p(np.ascontiguousarray(u, dtype=np.float64)), _p(y)) == 0
        return y

    def a12_avx_raw(self, p):
        y = np.zeros(self._coords.size)
        assert self.L.ref_a12_avx(_p(np.ascontiguousarray(p, dtype=np.float64)), _p(y)) == 0
        return y

    def marker_project(self, ptype, wil, xi, eta_p, rho_p, eta_q=None, rho_q=None):
        """Gauss-point (eta, rho) [27*nel] of the mesh given to setup() from
        markers, by the reference's projection ``ptype`` (src/rheology.c:150-185);
        eta_q / rho_q are the values on the Gauss points before the update."""
        nq = 27 * self.dims[0] * self.dims[1] * self.dims[2]
        eq = np.zeros(nq) if eta_q is None else np.array(eta_q, dtype=np.float64).reshape(-1)
        rq = np.zeros(nq) if rho_q is None else np.array(rho_q, dtype=np.float64).reshape(-1)
        w = np.ascontiguousarray(wil, dtype=np.int32)
        x = None if xi is None else np.ascontiguousarray(xi, dtype=np.float64).reshape(-1)
        rc = self.L.ref_marker_project(int(ptype), int(w.size), w.ctypes.data_as(C.POINTER(C.c_int32)),
                                       None if x is None else _p(x),
                                       _p(np.ascontiguousarray(eta_p, dtype=np.float64)),
                                       _p(np.ascontiguousarray(rho_p, dtype=np.float64)), _p(eq), _p(rq))
        assert rc == 0, rc
        return eq, rq

    def solcx_norms(self, eta0, eta1, xc, n, u, p):
        """[||v - v_ex||_L2, |E - E_ex|_H1s, H1, ||p - p_ex||_L2] of a discrete
        solution on the mesh given to setup() against the SolCx analytic
        solution, by the reference's Evaluate_uL2_symuH1_pL2 (src/inorms.c:188-363)
        and SolCxSolution (src/models/analytics_vv/SolCxSolution.c)."""
        out = np.zeros(4)
        rc = self.L.ref_solcx_norms(float(eta0), float(eta1), float(xc), int(n),
                                    _p(np.ascontiguousarray(u, dtype=np.float64)),
                                    _p(np.ascontiguousarray(p, dtype=np.float64)), _p(out))
        assert rc == 0, rc
        return out

    def solcx_exact(self, eta0, eta1, xc, n, pos):
        """SolCx analytic velocity [3] and pressure at pos [3]."""
        v, pr = np.zeros(3), np.zeros(1)
        rc = self.L.ref_solcx_exact(float(eta0), float(eta1), float(xc), int(n),
                                    _p(np.ascontiguousarray(pos, dtype=np.float64)), _p(v), _p(pr))
        assert rc == 0, rc
        return v, float(pr[0])

    def stokes_avx_raw(self, u, p):
        """MFStokesWrapper_A_AVX: [A11 u + A12 p; A21 u] without boundary conditions."""
        yu = np.zeros(self._coords.size)
        yp = np.zeros(4 * self.dims[0] * self.dims[1] * self.dims[2])
        assert self.L.ref_a_avx(_p(np.ascontiguousarray(u, dtype=np.float64)), _p(np.ascontiguousarray(p, dtype=np.float64)),
                                _p(yu), _p(yp)) == 0
        return yu, yp


# ------------------------------------------- material points -> Gauss points ---
# the reference's 3-point Gauss rule as it builds the volume quadrature, with
# 15-digit constants (QuadratureCreateGauss_3pnt_3D, src/quadrature.c:121-147)
_GP15 = np.array([-0.774596669241483, 0.0, 0.774596669241483])


def _q1_corner_weights(xi):
    """[..., 8] Q1 weights 0.125 (1 -+ xi)(1 -+ eta)(1 -+ zeta), corner bits (x, y, z)
    (pTatinConstructNI_Q1_3D, src/material_point_utils.c:502-519)."""
    xi = np.asarray(xi, dtype=np.float64)
    out = []
    for c in range(8):
        w = 0.125 * (1.0 + xi[..., 0] if c & 1 else 1.0 - xi[..., 0])
        w = w * (1.0 + xi[..., 1] if c & 2 else 1.0 - xi[..., 1])
        w = w * (1.0 + xi[..., 2] if c & 4 else 1.0 - xi[..., 2])
        out.append(w)
    return np.stack(out, axis=-1)


def _element_nodes(dims):
    """[nel, 27] lattice node index of every element node (x fastest)."""
    mx, my, mz = dims
    nx, ny = 2 * mx + 1, 2 * my + 1
    e = np.arange(mx * my * mz)
    ex, ey, ez = e % mx, (e // mx) % my, e // (mx * my)
    n = np.arange(27)
    a, b, c = n % 3, (n // 3) % 3, n // 9
    return (2 * ex[:, None] + a) + nx * ((2 * ey[:, None] + b) + ny * (2 * ez[:, None] + c))


_CORNER_NODES = np.array([0, 2, 6, 8, 18, 20, 24, 26])


def marker_project(dims, ptype, wil, xi, eta_p, rho_p, eta_q=None, rho_q=None, nodal=False):
    """Numpy restatement of the projection types of src/rheology.c:150-185 on a
    whole mesh: -1 keep, 0/10/20 P0 arithmetic/harmonic/geometric
    (src/material_point_utils.c:2567-2808), 1 Q1 (:604-801), 4 one-to-one
    (:803-840).  Returns Gauss-point (eta, rho) [27*nel]."""
    mx, my, mz = dims
    nel = mx * my * mz
    eq = np.zeros(27 * nel) if eta_q is None else np.array(eta_q, dtype=np.float64).reshape(-1)
    rq = np.zeros(27 * nel) if rho_q is None else np.array(rho_q, dtype=np.float64).reshape(-1)
    w = np.asarray(wil, dtype=np.int64)
    ve, vr = np.asarray(eta_p, dtype=np.float64), np.asarray(rho_p, dtype=np.float64)
    if ptype == -1:
        return eq, rq
    if ptype == 4:
        assert w.size == 27 * nel
        return ve.copy(), vr.copy()
    if ptype in (0, 10, 20):
        f = {0: ve, 10: 1.0 / ve, 20: np.log(ve)}[ptype]
        S, cnt, R = np.zeros(nel), np.zeros(nel), np.zeros(nel)
        np.add.at(S, w, f)
        np.add.at(cnt, w, 1.0)
        np.add.at(R, w, vr)
        with np.errstate(divide="ignore", invalid="ignore"):
            avg = {0: S / cnt, 10: cnt / S, 20: np.exp(S / cnt)}[ptype]
            return np.repeat(avg, 27), np.repeat(R / cnt, 27)
    if ptype != 1:
        raise ValueError(f"projection type {ptype} not supported")
    nn = (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1)
    nodes = _element_nodes(dims)
    A1, A2, B = np.zeros(nn), np.zeros(nn), np.zeros(nn)
    Nw = np.ones((w.size, 27))
    Nw[:, _CORNER_NODES] = _q1_corner_weights(np.asarray(xi, dtype=np.float64).reshape(-1, 3))
    g = nodes[w]
    np.add.at(A1, g, Nw * ve[:, None])
    np.add.at(A2, g, Nw * vr[:, None])
    np.add.at(B, g, Nw)
    nz = B != 0.0
    V1, V2 = np.zeros(nn), np.zeros(nn)
    V1[nz], V2[nz] = A1[nz] / B[nz], A2[nz] / B[nz]
    q = np.arange(27)
    xq = np.stack([_GP15[q % 3], _GP15[(q // 3) % 3], _GP15[q // 9]], axis=-1)
    Nq = _q1_corner_weights(xq)  # [27 points, 8 corners]
    out = []
    for V in (V1, V2):
        Ve = V[nodes]
        vals = Ve[:, _CORNER_NODES] @ Nq.T
        out.append(np.clip(vals, Ve.min(axis=1)[:, None], Ve.max(axis=1)[:, None]).reshape(-1))
    if nodal:  # also the nodal viscosity, the start of the type-1 coefficient hierarchy
        return out[0], out[1], V1
    return out[0], out[1]


# --------------------------------------------------- MatMult conventions ---
def matmult_a11(raw, x, mask):
    """MatMult_MFStokes_A11: zero Dirichlet columns, apply, y_k = x_k on Dirichlet rows."""
    xl = np.where(mask.astype(bool), 0.0, x)
    y = raw(xl)
    y[mask.astype(bool)] = x[mask.astype(bool)]
    return y


def matmult_a12(raw, p, mask):
    y = raw(p)
    y[mask.astype(bool)] = 0.0
    return y


def matmult_a21(raw, u, mask):
    return raw(np.where(mask.astype(bool), 0.0, u))


def get_diagonal(raw_diag, mask):
    d = raw_diag()
    d[mask.astype(bool)] = 1.0
    return d


# ------------------------------------------------------ dense Stokes solve ---
def body_force(R: Restatement, dims, coords, rho, g=(0.0, 0.0, -1.0)):
    R.L.o_body_force.argtypes = [C.c_int] * 3 + [_dp, _dp, C.c_double, C.c_double, C.c_double, _dp]
    bu = np.zeros(coords.size)
    R.L.o_body_force(*dims, _p(np.ascontiguousarray(coords, dtype=np.float64)),
                     _p(np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)), *map(float, g), _p(bu))
    return bu


def stokes_residual(R: Restatement, dims, coords, eta, mask, u, p, phi, fu, fp):
    """FormFunction_Stokes (src/stokes_form_function.c:477-564): insert the
    Dirichlet values phi into u, r_u = A11 u + A12 p - f_u, r_p = A21 u - f_p,
    then the Dirichlet rows r_k = u_k - phi_k (BCListResidualDirichlet, scale 1)."""
    for f in ("o_force_u", "o_force_p"):
        getattr(R.L, f).argtypes = [C.c_int] * 3 + [_dp] * 3
    m = mask.astype(bool)
    ub = np.where(m, phi, u)
    e = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(coords, dtype=np.float64)
    ru = R.a11_raw(dims, c, e, ub) + R.a12_raw(dims, c, p)
    bu = np.zeros(c.size)
    R.L.o_force_u(*dims, _p(c), _p(np.ascontiguousarray(fu, dtype=np.float64).reshape(-1)), _p(bu))
    ru -= bu
    rp = R.a21_raw(dims, c, ub)
    bp = np.zeros(rp.size)
    R.L.o_force_p(*dims, _p(c), _p(np.ascontiguousarray(fp, dtype=np.float64).reshape(-1)), _p(bp))
    rp -= bp
    ru[m] = u[m] - phi[m]
    return ru, rp


def stokes_dense(R: Restatement, dims, coords, eta, mask):
    """Assemble [A11 A12; A21 0] with the MatMult boundary convention by probing
    the oracle operators column by column (small meshes only)."""
    nu = coords.size
    nel = dims[0] * dims[1] * dims[2]
    npr = 4 * nel
    e = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1)
    m = mask.astype(bool)
    K = np.zeros((nu + npr, nu + npr))
    for j in range(nu):
        x = np.zeros(nu)
        x[j] = 1.0
        K[:nu, j] = matmult_a11(lambda v: R.a11_raw(dims, coords, e, v), x, mask)
        K[nu:, j] = matmult_a21(lambda v: R.a21_raw(dims, coords, v), x, mask)
    for j in range(npr):
        p = np.zeros(npr)
        p[j] = 1.0
        K[:nu, nu + j] = matmult_a12(lambda v: R.a12_raw(dims, coords, v), p, mask)
    return K


def stokes_dense_solve(R: Restatement, dims, coords, eta, mask, bu, bp=None):
    K = stokes_dense(R, dims, coords, eta, mask)
    nel = dims[0] * dims[1] * dims[2]
    b = np.concatenate([bu, np.zeros(4 * nel) if bp is None else bp])
    x = np.linalg.solve(K, b)
    return x[:coords.size], x[coords.size:]
