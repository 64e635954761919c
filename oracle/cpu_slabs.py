"""Slab-partitioned CPU MatMult of the reference kernel (CPU baseline only; the
product never imports it).

P processes, one per host core, each apply the reference's own
MFStokesWrapper_A11_AVX (oracle/_ref, one OpenMP thread) to a z-slab of the
elements, the way the reference runs one MPI rank per core on a DMDA
decomposition (src/stokes_operators.c:1171-1193); it avoids the `omp critical`
scatter of the threaded kernel.  The processes start together at a barrier and
the apply time is the slowest slab's.  The node plane two slabs share is
summed by the ranks' halo exchange in the reference; that sum is not timed.
"""
from __future__ import annotations

import multiprocessing as mp
import time
from multiprocessing import shared_memory

import numpy as np


def _worker(names, shapes, m, z0, z1, steps, warmup, barrier, out_q, rank, collect):
    from oracle.oracle import Reference
    shm = [shared_memory.SharedMemory(name=n) for n in names]
    try:
        coords, eta, x = (np.ndarray(s, dtype=np.float64, buffer=b.buf) for s, b in zip(shapes, shm))
        P = 3 * (2 * m + 1) ** 2  # values of one node plane
        c = coords[2 * z0 * P:(2 * z1 + 1) * P].copy()
        e = eta[z0 * m * m:z1 * m * m].copy()
        xs = x[2 * z0 * P:(2 * z1 + 1) * P].copy()
        F = Reference()
        F.setup((m, m, z1 - z0), c, e)
        F.set_threads(1)
        y = np.zeros_like(xs)
        for _ in range(warmup):
            F.a11_raw(xs, "avx", out=y)
        barrier.wait()
        t0 = time.perf_counter()
        for _ in range(steps):
            F.a11_raw(xs, "avx", out=y)
        dt = (time.perf_counter() - t0) / max(1, steps)
        if collect:
            y[...] = 0.0
            F.a11_raw(xs, "avx", out=y)
        out_q.put((rank, dt, y if collect else None))
    finally:
        for b in shm:
            b.close()


def slab_apply_time(coords, eta, x, m, nproc, steps=5, warmup=1, timeout=600, collect=False):
    """Seconds per apply of the whole m^3 mesh cut into nproc z-slabs; with
    collect, also the assembled result (the slabs' partial sums added on the
    node planes they share)."""
    nproc = max(1, min(nproc, m))
    arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in (coords, np.asarray(eta).reshape(-1, 27), x)]
    shm = []
    try:
        for a in arrays:
            b = shared_memory.SharedMemory(create=True, size=a.nbytes)
            np.ndarray(a.shape, dtype=np.float64, buffer=b.buf)[...] = a
            shm.append(b)
        ctx = mp.get_context("spawn")
        barrier = ctx.Barrier(nproc)
        q = ctx.Queue()
        cuts = [round(r * m / nproc) for r in range(nproc + 1)]
        procs = [ctx.Process(target=_worker, args=([b.name for b in shm], [a.shape for a in arrays], m, cuts[r],
                                                   cuts[r + 1], steps, warmup, barrier, q, r, collect))
                 for r in range(nproc)]
        for p in procs:
            p.start()
        times, parts, t_end = [], {}, time.monotonic() + timeout
        try:
            while len(times) < nproc:
                try:
                    rank, dt, ys = q.get(timeout=1.0)
                    times.append(dt)
                    parts[rank] = ys
                except Exception:  # queue empty: stop if a worker died or time ran out
                    if any(p.exitcode not in (None, 0) for p in procs) or time.monotonic() > t_end:
                        raise RuntimeError("slab worker failed or timed out")
        finally:
            for p in procs:
                p.join(timeout=10)
                if p.is_alive():
                    p.terminate()
        if not collect:
            return max(times)
        P = 3 * (2 * m + 1) ** 2
        y = np.zeros(arrays[2].size)
        for r, ys in parts.items():
            y[2 * cuts[r] * P:(2 * cuts[r + 1] + 1) * P] += ys
        return max(times), y
    finally:
        for b in shm:
            b.close()
            b.unlink()
