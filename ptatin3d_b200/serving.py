"""Solve server: continuous admission of independent Stokes solves.

A thin front end of p3d_server_* (include/p3d_b200.h): requests of uneven
mesh sizes are queued, admitted first-in first-out as execution slots and
device memory free up, and run concurrently on the device, each with its
solver state resident in HBM; results come back with their queueing and
end-to-end latencies.  Host arrays of a request are kept alive here until its
result has been returned.
"""
from __future__ import annotations

import ctypes as C
import itertools

import numpy as np

from ._lib import P3D_ERR_TIMEOUT, P3D_OK, Request, Result, ServerStats, check, lib
from .solver import default_opts


class StokesServer:
    def __init__(self, device: int = 0, hbm_budget: int = 16 << 30, max_active: int = 4, group_max: int = 8,
                 group_elements: int = 16384, group_overtake_ms: int = 2000):
        """group_max: requests of one shape solved together in a rolling
        group (shared launches; later arrivals join at restart boundaries,
        members leave when done); 1 solves every request on its own.
        group_elements: meshes with more elements are solved alone.
        group_overtake_ms: a request is grouped ahead of queued requests of
        other shapes only if none of them arrived that much earlier."""
        import torch  # noqa: F401  (the server shares the process's CUDA context)
        h = C.c_void_p()
        check(lib().p3d_server_create(int(device), int(hbm_budget), int(max_active), C.byref(h)))
        self.h = h
        check(lib().p3d_server_set_group_max(h, int(group_max)))
        check(lib().p3d_server_set_group_elements(h, int(group_elements)))
        check(lib().p3d_server_set_group_overtake_ms(h, int(group_overtake_ms)))
        self._live = {}
        self._tags = itertools.count()

    def submit(self, dims, dirichlet, coords, eta, rho, g=(0.0, 0.0, -1.0), tag=None, **opts) -> int:
        mx, my, mz = dims
        nn = (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1)
        nel = mx * my * mz
        arrs = dict(coords=np.ascontiguousarray(coords, dtype=np.float64).reshape(-1),
                    eta=np.ascontiguousarray(eta, dtype=np.float64).reshape(-1),
                    rho=np.ascontiguousarray(rho, dtype=np.float64).reshape(-1),
                    u=np.zeros(3 * nn), p=np.zeros(4 * nel))
        if arrs["coords"].size != 3 * nn or arrs["eta"].size != 27 * nel or arrs["rho"].size != 27 * nel:
            raise ValueError("request arrays do not match the mesh")
        tag = next(self._tags) if tag is None else int(tag)
        r = Request(mx, my, mz, int(dirichlet), arrs["coords"].ctypes.data, arrs["eta"].ctypes.data,
                    arrs["rho"].ctypes.data, float(g[0]), float(g[1]), float(g[2]), arrs["u"].ctypes.data,
                    arrs["p"].ctypes.data, default_opts(**opts), tag)
        self._live[tag] = arrs
        check(lib().p3d_server_submit(self.h, C.byref(r)))
        return tag

    def poll(self, timeout_ms: int = 0, max_results: int = 64):
        buf = (Result * max_results)()
        n = C.c_int32()
        rc = lib().p3d_server_poll(self.h, buf, max_results, int(timeout_ms), C.byref(n))
        if rc == P3D_ERR_TIMEOUT:  # nothing finished within timeout_ms
            return []
        check(rc)
        out = []
        for r in buf[:n.value]:
            arrs = self._live.pop(r.tag)
            out.append(dict(tag=r.tag, status=r.status, ok=r.status == P3D_OK, iterations=r.iterations,
                            rel_residual=r.rel_residual, wait_ms=r.wait_ms, run_ms=r.run_ms,
                            latency_ms=r.latency_ms, u=arrs["u"], p=arrs["p"]))
        return out

    def cancel(self, tag: int) -> None:
        """Cancel a queued or running request; its result (status
        P3D_ERR_CANCELLED) still comes back through poll."""
        check(lib().p3d_server_cancel(self.h, int(tag)))

    def wait_all(self, timeout_ms: int = 100):
        res = []
        while self._live:
            res += self.poll(timeout_ms)
        return res

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().p3d_server_get_stats(self.h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().p3d_server_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
