"""Failure paths of the solver and the solve server, provoked on the host (no
GPU fault is ever made): bad coefficients in one request, cancellation, an
exhausted device (allocation failures injected in the library's allocator)
and the poll timeout.  The reference exits the process on any CUDA error
(src/stokes_operators_cuda.cu:46-57); here every failure comes back as a
status, and the other work in flight is unaffected."""
import ctypes as C
import time

import numpy as np
import pytest
import torch

from cases import rel
from ptatin3d_b200 import PREC_F32, SCHUR_ETA_GEOMEAN, P3DError
from ptatin3d_b200 import _lib
from ptatin3d_b200 import mesh as M
from ptatin3d_b200.serving import StokesServer
from ptatin3d_b200.solver import StokesSolver, max_levels

pytestmark = pytest.mark.gpu
BITS = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
OPTS = dict(rtol=1e-11, max_it=3000, schur_eta=SCHUR_ETA_GEOMEAN, mg_precision=PREC_F32)


def request(m, nsph, contrast, seed):
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(nsph, seed, 0.15)
    return c, M.sinker_eta(qp, cen, r, 1.0, contrast), M.sinker_density(qp, cen, r, 1.0, 1.01)


def submit(S, m, arrays, tag, **kw):
    return S.submit((m, m, m), BITS, *arrays, tag=tag, nlevels=max_levels(m), **dict(OPTS, **kw))


@pytest.fixture
def no_injection():
    yield
    _lib.lib().p3d_debug_fail_allocations_after(-1)


def test_bad_requests_fail_alone_and_leave_the_others_unchanged(cuda):
    """A NaN in one request's viscosity (caught when the multigrid diagonal
    and spectrum are set up) and a NaN in another's density (a non-finite
    residual in the solve) return P3D_ERR_BREAKDOWN, while the three good
    requests solved beside them give the solutions they give alone."""
    good = {t: (m, request(m, ns, cst, 20 + t)) for t, (m, ns, cst) in enumerate([(8, 2, 1e2), (12, 3, 1e2), (16, 1, 10.0)])}
    alone = {}
    with StokesServer(hbm_budget=8 << 30, max_active=1) as S:
        for t, (m, arr) in good.items():
            submit(S, m, arr, t)
            alone[t] = S.wait_all()[0]
    assert all(r["ok"] for r in alone.values())
    c, eta, rho = request(12, 2, 1e2, 7)
    eta_nan = eta.copy()
    eta_nan[5, 3] = np.nan
    rho_nan = rho.copy()
    rho_nan[9, 0] = np.nan
    with StokesServer(hbm_budget=8 << 30, max_active=4) as S:
        submit(S, 12, (c, eta_nan, rho), 100)
        for t, (m, arr) in good.items():
            submit(S, m, arr, 10 + t)
        submit(S, 12, (c, eta, rho_nan), 101)
        res = {r["tag"]: r for r in S.wait_all()}
        st = S.stats()
    assert res[100]["status"] == _lib.P3D_ERR_BREAKDOWN
    assert res[101]["status"] == _lib.P3D_ERR_BREAKDOWN
    for t in good:
        assert res[10 + t]["ok"], res[10 + t]["status"]
        assert rel(res[10 + t]["u"], alone[t]["u"]) <= 1e-7
        assert rel(res[10 + t]["p"], alone[t]["p"]) <= 1e-6
    assert st["completed"] == 5 and st["active"] == 0


def test_solver_setup_rejects_nan_viscosity(cuda):
    m = 8
    c, eta, rho = request(m, 2, 1e2, 3)
    eta[0, 0] = np.nan
    S = StokesSolver(m, m, m, BITS, nlevels=3)
    try:
        with pytest.raises(P3DError) as e:
            S.setup(c, eta)
        assert e.value.code == _lib.P3D_ERR_BREAKDOWN
    finally:
        S.destroy()


def test_cancel_queued_and_running_requests(cuda):
    """With one execution slot, a long solve runs and a second request
    queues.  Cancelling the queued one completes it at once; cancelling the
    running one ends it after its current outer iteration.  Both come back
    P3D_ERR_CANCELLED, the slot is free again and the next request solves."""
    long_req = request(32, 8, 1e5, 5)
    small = request(8, 2, 1e2, 6)
    with StokesServer(hbm_budget=8 << 30, max_active=1) as S:
        submit(S, 32, long_req, 1, rtol=1e-14, max_it=100000)
        submit(S, 8, small, 2)
        t0 = time.perf_counter()
        while S.stats()["active"] == 0:  # the long solve is admitted (bounded wait)
            assert time.perf_counter() - t0 < 60
            time.sleep(0.01)
        S.cancel(2)
        first = S.poll(timeout_ms=5000)
        assert [r["tag"] for r in first] == [2] and first[0]["status"] == _lib.P3D_ERR_CANCELLED
        time.sleep(0.3)
        S.cancel(1)
        res = S.wait_all()
        assert len(res) == 1 and res[0]["tag"] == 1 and res[0]["status"] == _lib.P3D_ERR_CANCELLED
        assert res[0]["iterations"] < 100000  # stopped long before its limit
        with pytest.raises(P3DError):
            S.cancel(1)  # finished: nothing to cancel
        submit(S, 8, small, 3)
        after = S.wait_all()
        assert after[0]["ok"]
        st = S.stats()
        assert st["active"] == 0 and st["queued"] == 0 and st["completed"] == 3


def test_allocation_failures_return_nomem_without_leaks(cuda, no_injection):
    """Device allocations that fail (injected after a number of successful
    ones) make p3d_solver_create and a served request return P3D_ERR_NOMEM;
    everything allocated before the failure is given back, and once the
    device has memory again the same work succeeds."""
    L = _lib.lib()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for after in (0, 3, 8):  # p3d_solver_create makes 12 device allocations
        L.p3d_debug_fail_allocations_after(after)
        with pytest.raises(P3DError) as e:
            StokesSolver(16, 16, 16, BITS, nlevels=3)
        assert e.value.code == _lib.P3D_ERR_NOMEM
    L.p3d_debug_fail_allocations_after(-1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 <= 4 << 20  # nothing held back (allocation granularity aside)
    arr = request(12, 2, 1e2, 8)
    with StokesServer(hbm_budget=8 << 30, max_active=2) as S:
        L.p3d_debug_fail_allocations_after(5)  # the request's slot creation runs out
        submit(S, 12, arr, 1)
        r = S.wait_all()[0]
        assert r["status"] == _lib.P3D_ERR_NOMEM
        st = S.stats()
        assert st["device_bytes"] == 0 and st["active"] == 0  # its memory reservation was returned
        L.p3d_debug_fail_allocations_after(-1)
        submit(S, 12, arr, 2)
        assert S.wait_all()[0]["ok"]


def test_poll_times_out_when_nothing_finishes(cuda):
    L = _lib.lib()
    h = C.c_void_p()
    _lib.check(L.p3d_server_create(0, 1 << 30, 1, C.byref(h)))
    try:
        buf = (_lib.Result * 4)()
        n = C.c_int32(-1)
        t0 = time.perf_counter()
        assert L.p3d_server_poll(h, buf, 4, 50, C.byref(n)) == _lib.P3D_ERR_TIMEOUT
        assert n.value == 0 and time.perf_counter() - t0 >= 0.045
        assert L.p3d_server_poll(h, buf, 4, 0, C.byref(n)) == _lib.P3D_OK and n.value == 0
    finally:
        L.p3d_server_destroy(h)
