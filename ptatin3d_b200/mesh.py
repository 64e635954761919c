"""Structured Q2 meshes, viscosity fields and test vectors (numpy, host side).

Layouts follow the reference's ghosted local arrays for one process that owns
the whole mesh:
  coords / velocity : (nz, ny, nx, 3) node lattice flattened, x fastest,
                      nx = 2*mx+1 (src/dmda_element_q2p1.c:368-468)
  eta               : (nel, 27), element x fastest, q = qi + 3qj + 9qk
  pressure          : (nel, 4), P1disc [1, xh, yh, zh]

The generators reproduce the model constructions the reference's operator
tests use (viscous sinker on a Gaussian-bump mesh,
src/models/viscous_sinker/model_viscous_sinker_ops.c:56-128,668-690 and
src/mesh_deformation.c:48-131) and the seeded synthetic families the
benchmarks are quoted on (sinkers, layered, deformed log-normal).
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import FACE_IMAX, FACE_IMIN, FACE_JMAX, FACE_JMIN, FACE_KMAX, FACE_KMIN, bc_bit

GAUSS = np.array([-math.sqrt(0.6), 0.0, math.sqrt(0.6)])
GW = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
# Q2 Lagrange basis (nodes -1,0,1) at the Gauss points: BQ[q, a]
BQ = np.stack([0.5 * (GAUSS ** 2 - GAUSS), 1.0 - GAUSS ** 2, 0.5 * (GAUSS ** 2 + GAUSS)], axis=1)


def lattice_shape(mx, my, mz):
    return 2 * mz + 1, 2 * my + 1, 2 * mx + 1


def uniform_coords(mx, my, mz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """DMDASetUniformCoordinates on the Q2 node lattice: x_i = lo + i*(hi-lo)/(N-1)."""
    nz, ny, nx = lattice_shape(mx, my, mz)
    xs = lo[0] + np.arange(nx) * ((hi[0] - lo[0]) / (nx - 1))
    ys = lo[1] + np.arange(ny) * ((hi[1] - lo[1]) / (ny - 1))
    zs = lo[2] + np.arange(nz) * ((hi[2] - lo[2]) / (nz - 1))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X, Y, Z], axis=-1).reshape(-1)


def gaussian_bump_ymax(coords, mx, my, mz, amp=-0.3, lam=-5.6):
    """MeshDeformation_GaussianBump_YMAX (src/mesh_deformation.c:48-131): map the
    bounding box to [-1,1]^3, set y_j = -1 + j*(h(x,z)+1)/(MY-1) with
    h = amp*exp(lam*(x^2+z^2)) + 1, then map back to the bounding box."""
    nz, ny, nx = lattice_shape(mx, my, mz)
    c = coords.reshape(nz, ny, nx, 3)
    gmin = c.reshape(-1, 3).min(axis=0)
    gmax = c.reshape(-1, 3).max(axis=0)
    xs = -1.0 + np.arange(nx) * (2.0 / (nx - 1))
    ys = -1.0 + np.arange(ny) * (2.0 / (ny - 1))
    zs = -1.0 + np.arange(nz) * (2.0 / (nz - 1))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    height = amp * np.exp(lam * (X * X + Z * Z)) + 1.0
    dy = (height + 1.0) / (ny - 1)
    J = np.arange(ny)[None, :, None] * np.ones((nz, ny, nx))
    Yn = -1.0 + J * dy
    out = np.empty((nz, ny, nx, 3))
    out[..., 0] = (gmax[0] - gmin[0]) * (X + 1.0) / 2.0 + gmin[0]
    out[..., 1] = (gmax[1] - gmin[1]) * (Yn + 1.0) / 2.0 + gmin[1]
    out[..., 2] = (gmax[2] - gmin[2]) * (Z + 1.0) / 2.0 + gmin[2]
    return out.reshape(-1)


def perturb_interior(coords, mx, my, mz, frac=0.2, seed=0):
    """Move every interior lattice node by U[-frac*h, frac*h] per coordinate,
    h = lattice spacing (half an element), seeded."""
    nz, ny, nx = lattice_shape(mx, my, mz)
    c = coords.reshape(nz, ny, nx, 3).copy()
    rng = np.random.default_rng(seed)
    h = np.array([1.0 / (nx - 1), 1.0 / (ny - 1), 1.0 / (nz - 1)])
    d = rng.uniform(-frac, frac, size=(nz - 2, ny - 2, nx - 2, 3)) * h
    c[1:-1, 1:-1, 1:-1, :] += d
    return c.reshape(-1)


def _hash_uniform(idx, seed):
    """Counter-based U[-1, 1) from integer indices (splitmix64 finaliser)."""
    with np.errstate(over="ignore"):
        z = (idx.astype(np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)) * np.uint64(0xBF58476D1CE4E5B9)
        z ^= z >> np.uint64(27)
        z *= np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def slab_coords(mx, my, mz_global, z0, z1, frac=0.2, seed=0):
    """Coordinates of element layers [z0, z1) of an mx*my*mz_global unit-cube
    mesh whose interior lattice nodes are moved by U[-frac*h, frac*h] per
    coordinate.  The displacement of a node is a hash of its global lattice
    index, so slabs of different ranks agree on the node planes they share
    and the union of all slabs is one consistent mesh."""
    nx, ny, nzg = 2 * mx + 1, 2 * my + 1, 2 * mz_global + 1
    k = np.arange(2 * z0, 2 * z1 + 1)
    K, J, I = np.meshgrid(k, np.arange(ny), np.arange(nx), indexing="ij")
    h = np.array([1.0 / (nx - 1), 1.0 / (ny - 1), 1.0 / (nzg - 1)])
    c = np.stack([I * h[0], J * h[1], K * h[2]], axis=-1)
    g = (I + nx * (J + ny * K.astype(np.int64))).astype(np.int64)
    interior = (I > 0) & (I < nx - 1) & (J > 0) & (J < ny - 1) & (K > 0) & (K < nzg - 1)
    for l in range(3):
        d = _hash_uniform(3 * g + l, seed) * frac * h[l]
        c[..., l] += np.where(interior, d, 0.0)
    return c.reshape(-1)


def qp_coords(coords, mx, my, mz):
    """Physical coordinates of the 27 Gauss points of every element: (nel, 27, 3)."""
    nz, ny, nx = lattice_shape(mx, my, mz)
    c = coords.reshape(nz, ny, nx, 3)
    # gather element node blocks along x: (nz, ny, mx, 3a, 3)
    bx = np.stack([c[:, :, a:a + 2 * mx:2, :] for a in range(3)], axis=3)
    tx = np.einsum("qa,zymad->zymqd", BQ, bx)  # (nz, ny, mx, 3qi, 3)
    by = np.stack([tx[:, b:b + 2 * my:2] for b in range(3)], axis=2)  # (nz, my, 3b, mx, 3qi, 3)
    ty = np.einsum("qb,zmbxid->zmqxid", BQ, by)  # (nz, my, 3qj, mx, 3qi, 3)
    bz = np.stack([ty[c0:c0 + 2 * mz:2] for c0 in range(3)], axis=1)  # (mz, 3c, my, 3qj, mx, 3qi, 3)
    tz = np.einsum("kc,zcyjxid->zkyjxid", BQ, bz)  # (mz, 3qk, my, 3qj, mx, 3qi, 3)
    out = tz.transpose(0, 2, 4, 1, 3, 5, 6)  # (mz, my, mx, qk, qj, qi, 3)
    return np.ascontiguousarray(out).reshape(mx * my * mz, 27, 3)


def sinker_eta(qp, centres, radius, eta0=1.0, eta1=1e3):
    """eta = eta1 inside any sphere, eta0 elsewhere, evaluated at Gauss points."""
    eta = np.full(qp.shape[:2], eta0)
    for cc in np.atleast_2d(centres):
        inside = np.sum((qp - cc) ** 2, axis=-1) <= radius * radius
        eta[inside] = eta1
    return eta


def sinker_density(qp, centres, radius, rho0=1.0, rho1=1.01):
    rho = np.full(qp.shape[:2], rho0)
    for cc in np.atleast_2d(centres):
        rho[np.sum((qp - cc) ** 2, axis=-1) <= radius * radius] = rho1
    return rho


def random_sinkers(n, seed, radius=0.1):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, size=(n, 3)), radius


def layered_eta(qp, seed, nlayers=6, ninclusions=16, lo=-3.0, hi=3.0):
    """log10 eta uniform in [lo,hi] per horizontal (z) layer plus random
    spherical inclusions (radius U[0.05,0.15], log10 eta U[lo,hi])."""
    rng = np.random.default_rng(seed)
    layer_val = rng.uniform(lo, hi, size=nlayers)
    z = qp[..., 2]
    idx = np.clip((z * nlayers).astype(int), 0, nlayers - 1)
    leta = layer_val[idx]
    cen = rng.uniform(0.0, 1.0, size=(ninclusions, 3))
    rad = rng.uniform(0.05, 0.15, size=ninclusions)
    val = rng.uniform(lo, hi, size=ninclusions)
    for cc, r, v in zip(cen, rad, val):
        leta[np.sum((qp - cc) ** 2, axis=-1) <= r * r] = v
    return 10.0 ** leta


def lognormal_grf_eta(mx, my, mz, seed, sigma_decades=2.0, corr_len=0.1):
    """Per-element log-normal viscosity: log10 eta = sigma * g, g a unit-variance
    Gaussian random field with Gaussian covariance of length corr_len, built by
    FFT filtering of seeded white noise on the element grid; median 1."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((mz, my, mx))
    kz = np.fft.fftfreq(mz)[:, None, None] * mz
    ky = np.fft.fftfreq(my)[None, :, None] * my
    kx = np.fft.fftfreq(mx)[None, None, :] * mx
    k2 = (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2)
    filt = np.exp(-0.25 * k2 * corr_len ** 2)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g = (g - g.mean()) / (g.std() + 1e-300)
    eta_el = 10.0 ** (sigma_decades * g)
    return np.repeat(eta_el.reshape(-1, 1), 27, axis=1)


# ------------------------------------------------------------ boundary ----
FREE_SLIP = (bc_bit(FACE_IMIN, 0) | bc_bit(FACE_IMAX, 0) | bc_bit(FACE_JMIN, 1) | bc_bit(FACE_JMAX, 1)
             | bc_bit(FACE_KMIN, 2) | bc_bit(FACE_KMAX, 2))
# viscous sinker VSBC_FreeSlipFreeSurface (model_viscous_sinker_ops.c:236-244): no jmax
FREE_SLIP_FREE_SURFACE = (bc_bit(FACE_IMIN, 0) | bc_bit(FACE_IMAX, 0) | bc_bit(FACE_JMIN, 1)
                          | bc_bit(FACE_KMIN, 2) | bc_bit(FACE_KMAX, 2))
NO_SLIP = sum(bc_bit(f, c) for f in range(6) for c in range(3))


def dirichlet_mask(mx, my, mz, bits):
    """uint8 mask over the 3*nn velocity dofs from a face/component bit set."""
    nz, ny, nx = lattice_shape(mx, my, mz)
    m = np.zeros((nz, ny, nx, 3), dtype=np.uint8)
    faces = {FACE_IMIN: (slice(None), slice(None), 0), FACE_IMAX: (slice(None), slice(None), nx - 1),
             FACE_JMIN: (slice(None), 0, slice(None)), FACE_JMAX: (slice(None), ny - 1, slice(None)),
             FACE_KMIN: (0, slice(None), slice(None)), FACE_KMAX: (nz - 1, slice(None), slice(None))}
    for f, sl in faces.items():
        for comp in range(3):
            if bits & bc_bit(f, comp):
                m[sl + (comp,)] = 1
    return m.reshape(-1)


# ------------------------------------------------------------- vectors ----
def test_vector_velocity(coords):
    """_GenerateTestVector (src/tests/test_stokes_operators.c:48-92): u_d = X+Y+Z+d+3."""
    c = coords.reshape(-1, 3)
    s = c.sum(axis=1)
    return np.stack([s + 3.0, s + 4.0, s + 5.0], axis=1).reshape(-1)


def test_vector_pressure(mx, my, mz):
    """_GenerateTestVectorDAP (src/tests/test_stokes_operators.c:94-137) on the
    element-major P1disc layout: p_d = (-1+i*dx)+(-1+j*dy)+(-1+k*dz)+d+3,
    dx = 2/(M-1) (inf/nan for a single element in a direction, as in the reference)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        dx = 2.0 / np.float64(mx - 1)
        dy = 2.0 / np.float64(my - 1)
        dz = 2.0 / np.float64(mz - 1)
        K, J, I = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
        base = (-1.0 + I * dx) + (-1.0 + J * dy) + (-1.0 + K * dz)
        return np.stack([base + d + 3.0 for d in range(4)], axis=-1).reshape(-1)
