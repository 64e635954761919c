"""CPU restatement of the device Stokes solver (TEST INFRASTRUCTURE and the
CPU solve baseline of bench.py only; the product never imports it).

The same algorithm as the device solve, on host cores:

* outer FGMRES(m), right preconditioned, two-pass classical Gram-Schmidt (the
  device skips the second pass when the first removed less than half of the
  vector's norm squared; the basis is the same up to rounding);
* block upper-triangular preconditioner: z_p = S^-1 r_p with the per-element
  4x4 viscosity-scaled pressure mass matrix
  (src/stokes_assembly.c:299-450; element geometric-mean viscosity when
  ``schur_geomean``), then z_u = V-cycle(r_u - A12 z_p);
* V-cycle: Jacobi-preconditioned Chebyshev(k) on [lo, hi] * lambda_max(D^-1 A)
  (lambda_max from CG-Lanczos), Dirichlet-masked trilinear lattice transfers
  (the DMDA interpolation of src/ptatin_driver_linear_ts.c:986-990), Galerkin
  coarse operators P^T A P (OP_TYPE_GALERKIN, :712-762), the coarsest level
  inverted densely.

The fine-level operators are the reference's own compiled kernels, the ones
its AVX back end calls (oracle/_ref): MFStokesWrapper_A11_AVX (OpenMP) in the
smoother, MFStokesWrapper_A_AVX for the outer operator, MFStokesWrapper_A12_AVX
in the preconditioner and the diagonal of src/stokes_operators_mf.c, under the
MatMult conventions of src/stokes_operators.c.  The Galerkin levels are scipy
sparse matrices formed by probing the fine operator with 27 colours x 3
components.
"""
from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sp

from .oracle import Reference, Restatement, body_force, get_diagonal, matmult_a11, matmult_a12


def lattice_mask(n, bits):
    """Dirichlet flags of a node lattice n = (nx, ny, nz), 3 interleaved
    components; bit 3*face + comp, faces imin, imax, jmin, jmax, kmin, kmax."""
    nx, ny, nz = n
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    faces = [i == 0, i == nx - 1, j == 0, j == ny - 1, k == 0, k == nz - 1]
    mask = np.zeros((nz, ny, nx, 3), dtype=bool)
    for f, on in enumerate(faces):
        for c in range(3):
            if (bits >> (3 * f + c)) & 1:
                mask[..., c] |= on
    return mask.reshape(-1)


def _interp_1d(nc):
    nf = 2 * nc - 1
    rows, cols, vals = [], [], []
    for i in range(nf):
        if i % 2 == 0:
            rows.append(i); cols.append(i // 2); vals.append(1.0)
        else:
            rows += [i, i]; cols += [i // 2, i // 2 + 1]; vals += [0.5, 0.5]
    return sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))


def prolongation(nc, mask_f, mask_c):
    """Dirichlet-masked trilinear interpolation, coarse lattice nc -> fine (2nc-1)."""
    P = sp.kron(sp.kron(_interp_1d(nc[2]), _interp_1d(nc[1])), _interp_1d(nc[0]))
    P = sp.kron(P, sp.identity(3)).tocsr()
    return (sp.diags((~mask_f).astype(float)) @ P @ sp.diags((~mask_c).astype(float))).tocsr()


def _start_vector(n):
    """The device solver's deterministic start vector of the lambda_max
    estimate: xorshift64 (13, 7, 17) from 0x9E3779B97F4A7C15, the top 53 bits
    scaled to [0, 1), minus 1/2."""
    out = np.empty(n)
    st = 0x9E3779B97F4A7C15
    m64 = (1 << 64) - 1
    for i in range(n):
        st ^= (st << 13) & m64
        st ^= st >> 7
        st ^= (st << 17) & m64
        out[i] = (st >> 11) * (1.0 / 9007199254740992.0) - 0.5
    return out


def _lmax(A, dinv, mask, its=10):
    """lambda_max(D^-1 A) from CG-Lanczos, from the device solver's start vector."""
    r = _start_vector(dinv.size)
    r[mask] = 0.0
    z = dinv * r
    p = z.copy()
    rz = r @ z
    al, be = [], []
    for _ in range(its):
        q = A(p)
        pq = p @ q
        if not pq > 0:
            break
        a = rz / pq
        al.append(a)
        r = r - a * q
        z = dinv * r
        rz2 = r @ z
        b = rz2 / rz
        be.append(b)
        p = z + b * p
        rz = rz2
    m = len(al)
    T = np.zeros((m, m))
    for j in range(m):
        T[j, j] = 1.0 / al[j] + (be[j - 1] / al[j - 1] if j > 0 else 0.0)
        if j + 1 < m:
            T[j, j + 1] = T[j + 1, j] = np.sqrt(be[j]) / al[j]
    return float(np.linalg.eigvalsh(T).max())


class _Level:
    def __init__(self, n, mask, A, dinv):
        self.n, self.mask, self.A, self.dinv = n, mask, A, dinv
        self.lmax = None


class CpuStokesSolver:
    def __init__(self, m, coords, eta, rho, bits, nlevels=4, cheb_its=3, cheb_lo=0.2, cheb_hi=1.1, esteig=10,
                 restart=30, threads=None, schur_geomean=True, g=(0.0, 0.0, -1.0), inner_rtol=0.0, inner_its=0):
        t0 = time.perf_counter()
        self.inner_rtol, self.inner_its, self.inner_total = inner_rtol, inner_its, 0
        self.K, self.lo, self.hi, self.restart = cheb_its, cheb_lo, cheb_hi, restart
        dims = tuple(m) if isinstance(m, (tuple, list)) else (m, m, m)  # elements per direction
        nf = tuple(2 * d + 1 for d in dims)
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1)
        eta = np.ascontiguousarray(eta, dtype=np.float64).reshape(-1, 27)
        self.ref = Reference()
        self.ref.setup(dims, coords, eta)
        if threads:
            self.ref.set_threads(threads)
        mask = lattice_mask(nf, bits)
        mu8 = mask.astype(np.uint8)
        self.mask_u8 = mu8
        A0 = lambda v: matmult_a11(lambda w: self.ref.a11_raw(w, "avx"), v, mu8)
        fine = _Level(nf, mask, A0, 1.0 / get_diagonal(self.ref.diag_raw, mu8))
        levels = [fine]
        self.P = []
        # Galerkin hierarchy: level 1 by probing the matrix-free fine operator, then sparse triple products
        for lev in range(1, nlevels):
            F = levels[-1]
            nc = tuple((a + 1) // 2 for a in F.n)
            mc = lattice_mask(nc, bits)
            P = prolongation(nc, F.mask, mc)
            if lev == 1:
                Ac = self._probe_galerkin(F.A, P, nc, mc)
            else:
                Ac = (P.T @ F.Amat @ P).tocsr()
                Ac = Ac + sp.diags(mc.astype(float))  # identity rows on Dirichlet dofs
            Ac = Ac.tocsr()
            d = Ac.diagonal()
            L = _Level(nc, mc, (lambda M_: (lambda v: M_ @ v))(Ac), 1.0 / d)
            L.Amat = Ac
            self.P.append(P)
            levels.append(L)
        self.lv = levels[::-1]  # coarsest first
        self.P = self.P[::-1]   # P[l-1]: level l-1 -> l
        for L in self.lv[1:]:
            L.lmax = _lmax(L.A, L.dinv, L.mask, esteig)
        self.Acinv = np.linalg.inv(self.lv[0].Amat.toarray())
        # Schur blocks and right-hand side
        R = Restatement()
        e_s = eta
        if schur_geomean:
            e_s = np.repeat(np.exp(np.log(eta).mean(axis=1, keepdims=True)), 27, axis=1)
        self.Binv = np.linalg.inv(R.schur_mass(dims, coords, e_s.reshape(-1)))
        bu = body_force(R, dims, coords, np.asarray(rho, dtype=np.float64).reshape(-1), g)
        bu[mask] = 0.0
        self.nu, self.npr = coords.size, 4 * dims[0] * dims[1] * dims[2]
        self.b = np.concatenate([bu, np.zeros(self.npr)])
        self.setup_s = time.perf_counter() - t0

    @staticmethod
    def _probe_galerkin(A, P, nc, mc):
        """P^T A P as a 27-point block stencil: the coarse nodes of one colour
        (I, J, K mod 3) have at most one member in any 27-neighbourhood."""
        nx, ny, nz = nc
        K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        I, J, K = I.reshape(-1), J.reshape(-1), K.reshape(-1)
        nn = nx * ny * nz
        rows, cols, vals = [], [], []
        for ck in range(3):
            for cj in range(3):
                for ci in range(3):
                    member = (I % 3 == ci) & (J % 3 == cj) & (K % 3 == ck)
                    # for every node, the member of this colour among its neighbours
                    di = (ci - I % 3 + 3) % 3; di = np.where(di == 2, -1, di)
                    dj = (cj - J % 3 + 3) % 3; dj = np.where(dj == 2, -1, dj)
                    dk = (ck - K % 3 + 3) % 3; dk = np.where(dk == 2, -1, dk)
                    ok = (I + di >= 0) & (I + di < nx) & (J + dj >= 0) & (J + dj < ny) & (K + dk >= 0) & (K + dk < nz)
                    nb = (I + di) + nx * ((J + dj) + ny * (K + dk))
                    for d in range(3):
                        e = np.zeros(3 * nn)
                        e[3 * np.nonzero(member)[0] + d] = 1.0
                        e[mc] = 0.0
                        y = P.T @ A(P @ e)
                        for r in range(3):
                            rr = 3 * np.arange(nn) + r
                            cc = 3 * nb + d
                            sel = ok & ~mc[rr] & ~mc[np.where(ok, cc, 0)]
                            rows.append(rr[sel]); cols.append(cc[sel]); vals.append(y[rr[sel]])
        rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
        keep = vals != 0.0
        Ac = sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(3 * nn, 3 * nn))
        return (Ac + sp.diags(mc.astype(float))).tocsr()

    # -------------------------------------------------------------- V-cycle
    def _cheb(self, L, b, x=None):
        lo, hi = self.lo * L.lmax, self.hi * L.lmax
        th, de = 0.5 * (hi + lo), 0.5 * (hi - lo)
        sg = th / de
        if x is None:
            x = np.zeros_like(b)
            r = b.copy()
        else:
            r = b - L.A(x)
        d = L.dinv * r / th
        rho = 1.0 / sg
        for k in range(self.K):
            if k == self.K - 1:
                return x + d
            t = L.A(d)
            rn = 1.0 / (2.0 * sg - rho)
            x = x + d
            r = r - t
            d = rn * rho * d + 2.0 * rn / de * (L.dinv * r)
            rho = rn
        return x

    def vcycle(self, b, l=None):
        if l is None:
            l = len(self.lv) - 1
        if l == 0:
            bb = b.copy()
            bb[self.lv[0].mask] = 0.0
            return self.Acinv @ bb
        L, P = self.lv[l], self.P[l - 1]
        x = self._cheb(L, b)
        r = b - L.A(x)
        xc = self.vcycle(P.T @ r, l - 1)
        x = x + P @ xc
        return self._cheb(L, b, x)

    # --------------------------------------------------------------- FGMRES
    def op(self, x):
        """MatMult_MFStokes_A (src/stokes_operators.c:927, the AVX back end): Dirichlet
        columns of u zeroed, [A11 A12; A21 0] applied, Dirichlet rows y_k = u_k."""
        u, p = x[:self.nu], x[self.nu:]
        m = self.mask_u8.astype(bool)
        yu, yp = self.ref.stokes_avx_raw(np.where(m, 0.0, u), p)
        yu[m] = u[m]
        return np.concatenate([yu, yp])

    def velocity(self, b):
        """A11^-1 b: one V-cycle, or (inner_rtol > 0) conjugate gradients on
        A11 preconditioned by the V-cycle until |b - A x| <= inner_rtol |b| or
        inner_its iterations, in the device's order of operations (p starts at
        0 with rz_old = 1, so the first direction is z)."""
        if self.inner_rtol <= 0.0:
            return self.vcycle(b)
        A = self.lv[-1].A
        x, r, p = np.zeros_like(b), b.copy(), np.zeros_like(b)
        tol2 = self.inner_rtol ** 2 * (b @ b)
        rz_old, rr, k = 1.0, b @ b, 0
        while rr > tol2 and k < self.inner_its:
            z = self.vcycle(r)
            rz = r @ z
            p = z + (rz / rz_old) * p
            q = A(p)
            a = rz / (p @ q)
            x += a * p
            r -= a * q
            rr, rz_old, k = r @ r, rz, k + 1
        self.inner_total += k
        return x

    def pc(self, x):
        ru, rp = x[:self.nu], x[self.nu:]
        zp = np.einsum("eij,ej->ei", self.Binv, rp.reshape(-1, 4)).reshape(-1)
        t = ru - matmult_a12(self.ref.a12_avx_raw, zp, self.mask_u8)
        return np.concatenate([self.velocity(t), zp])

    def solve(self, rtol=1e-6, max_it=1000):
        """FGMRES from x = 0; returns (u, p, iterations, |r|/|r0|, seconds)."""
        t0 = time.perf_counter()
        b, m = self.b, self.restart
        x = np.zeros_like(b)
        its, r0, rel = 0, None, 1.0
        while its < max_it:
            r = b - self.op(x)
            beta = np.linalg.norm(r)
            if r0 is None:
                r0 = beta
            rel = beta / r0
            if beta <= rtol * r0:
                break
            V = np.zeros((m + 1, b.size))
            Z = np.zeros((m, b.size))
            V[0] = r / beta
            H = np.zeros((m + 1, m))
            g = np.zeros(m + 1)
            g[0] = beta
            cs, sn = np.zeros(m), np.zeros(m)
            j = 0
            while j < m and its < max_it:
                Z[j] = self.pc(V[j])
                w = self.op(Z[j])
                h = V[:j + 1] @ w
                w -= V[:j + 1].T @ h
                h2 = V[:j + 1] @ w
                w -= V[:j + 1].T @ h2
                H[:j + 1, j] = h + h2
                hn = np.linalg.norm(w)
                H[j + 1, j] = hn
                if hn > 0:
                    V[j + 1] = w / hn
                for i in range(j):
                    a_, b_ = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a_ + sn[i] * b_, -sn[i] * a_ + cs[i] * b_
                rr = np.hypot(H[j, j], H[j + 1, j])
                cs[j], sn[j] = (H[j, j] / rr, H[j + 1, j] / rr) if rr > 0 else (1.0, 0.0)
                H[j, j], H[j + 1, j] = rr, 0.0
                g[j + 1], g[j] = -sn[j] * g[j], cs[j] * g[j]
                its += 1
                j += 1
                rel = abs(g[j]) / r0
                if rel <= rtol or hn == 0.0:
                    break
            y = np.linalg.solve(np.triu(H[:j, :j]), g[:j])
            x = x + Z[:j].T @ y
            if rel <= rtol:
                break
        rt = np.linalg.norm(b - self.op(x)) / r0
        return x[:self.nu], x[self.nu:], its, rt, time.perf_counter() - t0
