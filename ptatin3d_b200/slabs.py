"""z-slab domain decomposition of the A11 apply across ranks.

The reference decomposes the DMDA over MPI ranks and wraps every matrix-free
MatMult in DMGlobalToLocal / DMLocalToGlobal(ADD) halo exchanges
(src/stokes_operators.c:1171-1172,1192-1193).  Here each rank owns a
contiguous range of element layers in z, [z0, z1), and keeps the node planes
2*z0 .. 2*z1 of its slab: the bottom and top planes are shared with the
neighbouring ranks.  One apply is

  1. the local element apply on the slab (Dirichlet columns zeroed, rows set,
     on the faces of the slab that lie on the global boundary),
  2. one exchange step: send the shared plane's partial sums to the
     neighbour, receive its partials and add them (point-to-point, NCCL over
     NVLink on GPUs, gloo on CPUs),
  3. Dirichlet rows on a shared plane reset to x (both ranks wrote them).

The local apply is passed in (`local_apply(x_slab, y_slab)`), so the same
exchange runs with the sm_100a operator on GPUs and with any CPU operator.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from ._lib import FACE_IMAX, FACE_IMIN, FACE_JMAX, FACE_JMIN, FACE_KMAX, FACE_KMIN, bc_bit


def slab_range(mz: int, rank: int, world: int):
    """Element layers [z0, z1) of rank `rank` (balanced contiguous split)."""
    base, rem = divmod(mz, world)
    z0 = rank * base + min(rank, rem)
    z1 = z0 + base + (1 if rank < rem else 0)
    return z0, z1


def slab_global_faces(rank: int, world: int) -> int:
    """Faces of the slab on the global boundary (bit f)."""
    f = (1 << FACE_IMIN) | (1 << FACE_IMAX) | (1 << FACE_JMIN) | (1 << FACE_JMAX)
    if rank == 0:
        f |= 1 << FACE_KMIN
    if rank == world - 1:
        f |= 1 << FACE_KMAX
    return f


def plane_dirichlet(mx, my, bits):
    """uint8 mask of one node plane (x fastest, 3 comps) from the x/y face bits."""
    nx, ny = 2 * mx + 1, 2 * my + 1
    m = np.zeros((ny, nx, 3), dtype=np.uint8)
    for face, sl in ((FACE_IMIN, (slice(None), 0)), (FACE_IMAX, (slice(None), nx - 1)),
                     (FACE_JMIN, (0, slice(None))), (FACE_JMAX, (ny - 1, slice(None)))):
        for c in range(3):
            if bits & bc_bit(face, c):
                m[sl + (c,)] = 1
    return m.reshape(-1)


class SlabExchange:
    """Shared-plane exchange of a slab-partitioned velocity vector."""

    def __init__(self, mx, my, mz, bits, rank=None, world=None, group=None, device=None):
        self.rank = dist.get_rank(group) if rank is None else rank
        self.world = dist.get_world_size(group) if world is None else world
        self.group = group
        self.mx, self.my, self.mz = mx, my, mz
        self.z0, self.z1 = slab_range(mz, self.rank, self.world)
        self.plane = 3 * (2 * mx + 1) * (2 * my + 1)
        self.nz_local = 2 * (self.z1 - self.z0) + 1
        self.n_local = self.plane * self.nz_local
        self.bits = bits
        m = plane_dirichlet(mx, my, bits).astype(bool)
        dev = device if device is not None else torch.device("cpu")
        self.plane_mask = torch.tensor(m, device=dev)

    def add_shared(self, x: torch.Tensor, y: torch.Tensor):
        """y[shared planes] += neighbour's partials; Dirichlet rows there reset to x."""
        P = self.plane
        ops, recv = [], []
        if self.rank > 0:
            rb = torch.empty(P, dtype=y.dtype, device=y.device)
            ops.append(dist.P2POp(dist.isend, y[:P].contiguous(), self.rank - 1, self.group))
            ops.append(dist.P2POp(dist.irecv, rb, self.rank - 1, self.group))
            recv.append((0, rb))
        if self.rank < self.world - 1:
            rt = torch.empty(P, dtype=y.dtype, device=y.device)
            ops.append(dist.P2POp(dist.isend, y[-P:].contiguous(), self.rank + 1, self.group))
            ops.append(dist.P2POp(dist.irecv, rt, self.rank + 1, self.group))
            recv.append((self.n_local - P, rt))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for off, buf in recv:
            if y.is_cuda:  # one library kernel: add the partials, reset the Dirichlet rows
                from ._lib import PREC_F32, PREC_F64, check, lib
                prec = PREC_F64 if y.dtype == torch.float64 else PREC_F32
                check(lib().p3d_slab_add_plane(prec, self.mx, self.my, self.bits, C.c_void_p(buf.data_ptr()),
                                               C.c_void_p(x[off:].data_ptr()), C.c_void_p(y[off:].data_ptr()),
                                               C.c_void_p(torch.cuda.current_stream(y.device).cuda_stream)))
            else:  # host ranks (gloo): the same arithmetic on CPU tensors
                seg = y[off:off + P]
                seg += buf
                xs = x[off:off + P]
                seg[self.plane_mask] = xs[self.plane_mask]


class SlabA11:
    """A11 MatMult on a z-slab partition: local apply + shared-plane exchange."""

    def __init__(self, exchange: SlabExchange, local_apply):
        self.ex = exchange
        self.local_apply = local_apply

    def mult(self, x_slab: torch.Tensor, y_slab: torch.Tensor):
        self.local_apply(x_slab, y_slab)
        self.ex.add_shared(x_slab, y_slab)


def device_slab_operator(mx, my, mz, bits, coords_slab, eta_slab, rank, world, precision=64, device=0):
    """The sm_100a operator of one slab with the MatMult boundary convention on
    the slab faces that lie on the global boundary."""
    from .operators import MatA11MF
    from ._lib import MeshDesc
    z0, z1 = slab_range(mz, rank, world)
    d = MeshDesc()
    d.mx, d.my, d.mz = mx, my, z1 - z0
    d.gx, d.gy, d.gz = 2 * mx + 1, 2 * my + 1, 2 * (z1 - z0) + 1
    d.ox = d.oy = d.oz = 0
    d.dirichlet = bits
    d.global_faces = slab_global_faces(rank, world)
    op = MatA11MF(d, precision, device)
    op.set_coefficients(coords_slab, eta_slab)
    return op
