"""z-slab decomposition of the A11 MatMult on 2 and 3 CPU ranks (gloo).

Each rank applies the operator of its slab (here the CPU oracle stands in for
the device operator: the code under test is the decomposition and the
shared-plane exchange) and the assembled result must equal the oracle's
global MatMult, Dirichlet rows on shared planes included.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ptatin3d_b200 import mesh as M
from ptatin3d_b200._lib import bc_bit
from ptatin3d_b200.slabs import SlabA11, SlabExchange, slab_global_faces, slab_range

DIMS = (3, 2, 7)
BITS = M.FREE_SLIP | bc_bit(M.FACE_IMIN, 1)


def _case():
    mx, my, mz = DIMS
    c = M.perturb_interior(M.uniform_coords(mx, my, mz), mx, my, mz, frac=0.15, seed=2)
    rng = np.random.default_rng(3)
    eta = 10.0 ** rng.uniform(-1, 1, size=(mx * my * mz, 27))
    x = rng.uniform(-1, 1, size=c.size)
    return c, eta, x


def _face_bits(faces):
    out = 0
    for f in range(6):
        if faces & (1 << f):
            out |= BITS & (7 << (3 * f))
    return out


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Restatement, matmult_a11
        R = Restatement()
        mx, my, mz = DIMS
        c, eta, x = _case()
        z0, z1 = slab_range(mz, rank, world)
        P = 3 * (2 * mx + 1) * (2 * my + 1)
        sl = slice(2 * z0 * P, (2 * z1 + 1) * P)
        c_s, x_s = c[sl], x[sl]
        e_s = eta.reshape(mz, my * mx, 27)[z0:z1].reshape(-1, 27)
        dims = (mx, my, z1 - z0)
        mask = M.dirichlet_mask(*dims, _face_bits(slab_global_faces(rank, world)))

        def local_apply(xt, yt):
            y = matmult_a11(lambda v: R.a11_raw(dims, c_s, e_s.reshape(-1), v), xt.numpy(), mask)
            yt.copy_(torch.from_numpy(y))

        ex = SlabExchange(mx, my, mz, BITS)
        op = SlabA11(ex, local_apply)
        xt = torch.tensor(x_s)
        yt = torch.empty_like(xt)
        op.mult(xt, yt)
        q.put((rank, z0, z1, yt.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_slab_matmult_matches_global(restatement, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mx, my, mz = DIMS
    c, eta, x = _case()
    from oracle.oracle import matmult_a11
    y_ref = matmult_a11(lambda v: restatement.a11_raw(DIMS, c, eta.reshape(-1), v), x, M.dirichlet_mask(*DIMS, BITS))
    P = 3 * (2 * mx + 1) * (2 * my + 1)
    for rank, z0, z1, y in res:
        ref = y_ref[2 * z0 * P:(2 * z1 + 1) * P]
        assert np.abs(y - ref).max() <= 1e-13 * np.abs(y_ref).max(), rank


def test_slab_ranges_cover_mesh():
    for mz in (1, 5, 16, 97):
        for world in (1, 2, 3, 8):
            if world > mz:
                continue
            rs = [slab_range(mz, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == mz
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1


def test_slab_coords_agree_on_shared_planes():
    """Hash-perturbed slabs form one mesh: shared planes match, the union is the global mesh."""
    mx, my, mzg = 3, 2, 7
    full = M.slab_coords(mx, my, mzg, 0, mzg, frac=0.2, seed=5).reshape(2 * mzg + 1, -1)
    P = 3 * (2 * mx + 1) * (2 * my + 1)
    for world in (2, 3):
        for r in range(world):
            z0, z1 = slab_range(mzg, r, world)
            s = M.slab_coords(mx, my, mzg, z0, z1, frac=0.2, seed=5).reshape(2 * (z1 - z0) + 1, -1)
            assert np.array_equal(s, full[2 * z0:2 * z1 + 1])
    # boundary nodes are not moved, interior nodes are, by at most 0.2 h
    u = M.uniform_coords(mx, my, mzg).reshape(2 * mzg + 1, -1)
    d = np.abs(full - u).reshape(2 * mzg + 1, 2 * my + 1, 2 * mx + 1, 3)
    assert d[0].max() == 0 and d[-1].max() == 0 and d[:, 0].max() == 0 and d[:, :, -1].max() == 0
    h = (1 / (2 * mx), 1 / (2 * my), 1 / (2 * mzg))
    for l in range(3):
        assert 0 < d[..., l].max() <= 0.2 * h[l] + 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_slab_plane_kernel_matches_host_arithmetic(cuda, dtype):
    """The library's receiving step of the shared-plane exchange
    (p3d_slab_add_plane: y += partials, Dirichlet rows reset to x) equals the
    host arithmetic the gloo ranks run."""
    import ctypes as C

    from ptatin3d_b200 import _lib
    from ptatin3d_b200.slabs import plane_dirichlet
    mx, my = 5, 3
    bits = M.FREE_SLIP
    P = 3 * (2 * mx + 1) * (2 * my + 1)
    g = torch.Generator().manual_seed(3)
    x, y, r = (torch.rand(P, generator=g, dtype=torch.float64) for _ in range(3))
    mask = torch.tensor(plane_dirichlet(mx, my, bits).astype(bool))
    ref = y + r
    ref[mask] = x[mask]
    xd, yd, rd = (t.to(device=cuda, dtype=dtype) for t in (x, y, r))
    prec = _lib.PREC_F64 if dtype == torch.float64 else _lib.PREC_F32
    _lib.check(_lib.lib().p3d_slab_add_plane(prec, mx, my, bits, C.c_void_p(rd.data_ptr()), C.c_void_p(xd.data_ptr()),
                                             C.c_void_p(yd.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    tol = 0.0 if dtype == torch.float64 else 1e-6
    assert float((yd.double().cpu() - ref).abs().max()) <= tol
