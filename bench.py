#!/usr/bin/env python
"""Benchmark of the matrix-free Q2 A11 apply (MatMult_MFStokes_A11 hot path).

Default workload: the FP64 A11 MatMult on the 96^3-element deformed mesh
(Q2, 7,189,057 nodes = 21,567,171 velocity dofs; interior lattice nodes
perturbed by U[-0.2h,0.2h]; per-element log-normal viscosity, sigma 2
decades, correlation length 0.1, seeded synthetic fields; free-slip walls).
A step is one apply of A11 to one velocity vector (every element, Dirichlet
columns/rows handled in the kernel).  Inputs (709 MB of algorithmic FP64
traffic per apply) exceed the 126 MB L2, so no L2 flush is needed between
steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N GPUs) the mesh is m x m x (m*N) elements cut into z-slabs
of m^3 elements, one per rank (weak scaling); a step applies every slab and
exchanges the node plane shared with each neighbour over NCCL, and `value`
is the dof throughput of the whole mesh, timed as the max over ranks.  `--impl reference`
times the reference's own CPU implementation of the same apply
(MFStokesWrapper_A11_AVX compiled from the pTatin3d sources into
oracle/_ref, all host threads) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "A11 MF apply GDoF/s (FP64, 96^3 Q2 deformed mesh)"
# the reference's flop count of one element apply (src/stokes_operators_cuda.cu:520-522)
REF_FLOPS_PER_EL = 17253
UNIT = "GDoF/s"


def workload(m=96, seed=4, kind="deformed"):
    """deformed: interior nodes perturbed, per-element log-normal eta (general geometry path);
    layered: uniform mesh, 6 layers of log10 eta in [-3,3] + 16 inclusions (affine path)."""
    from ptatin3d_b200 import mesh as M
    c = M.uniform_coords(m, m, m)
    if kind == "deformed":
        c = M.perturb_interior(c, m, m, m, frac=0.2, seed=seed)
        eta = M.lognormal_grf_eta(m, m, m, seed=seed, sigma_decades=2.0, corr_len=0.1)
    else:
        eta = M.layered_eta(M.qp_coords(c, m, m, m), seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=c.size)
    return dict(m=m, coords=c, eta=eta, x=x, bits=M.FREE_SLIP, kind=kind)


def metric_name(m, kind):
    """The metric of the apply line; the default workload gives METRIC."""
    return f"A11 MF apply GDoF/s (FP64, {m}^3 Q2 {kind} mesh)"


def workload_name(m, kind):
    if kind == "deformed":
        return (f"A11 MatMult, Q2 {m}^3 deformed mesh (interior nodes +-0.2h), log-normal eta "
                "(sigma 2 decades, corr 0.1), free-slip walls")
    return (f"A11 MatMult, Q2 {m}^3 uniform mesh, layered eta (6 layers, log10 eta in [-3,3], "
            "16 inclusions), free-slip walls")


def algorithmic_bytes(m, elem_bytes=8):
    """x read + y write + coords read + 27 eta per element (connectivity and
    Dirichlet mask are index arithmetic)."""
    nn = (2 * m + 1) ** 3
    return elem_bytes * (3 * nn + 3 * nn + 3 * nn + 27 * m ** 3)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return dist.get_rank(), world, local
    return 0, 1, 0


def reduce_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_apply(wl, steps, warmup, threads=None):
    """Time the reference's own A11 kernel (AVX backend, OpenMP) on the host."""
    from oracle.oracle import Reference, build
    if not Reference.available():
        build()
    F = Reference()
    m = wl["m"]
    F.setup((m, m, m), wl["coords"], wl["eta"])
    n = threads or os.cpu_count()
    F.set_threads(n)
    x = wl["x"]
    y = np.zeros_like(x)
    for _ in range(warmup):
        F.a11_raw(x, "avx", out=y)
    t0 = time.perf_counter()
    for _ in range(steps):
        F.a11_raw(x, "avx", out=y)
    dt = (time.perf_counter() - t0) / steps
    return dt, n


def cpu_slab_apply(wl, steps, warmup):
    """Time the reference's A11 kernel on z-slabs, one process (one thread) per
    host core, the way the reference runs one MPI rank per core."""
    from oracle.cpu_slabs import slab_apply_time
    from oracle.oracle import Reference, build
    if not Reference.available():
        build()
    n = min(os.cpu_count(), wl["m"])  # one element layer per process at least
    return slab_apply_time(wl["coords"], wl["eta"], wl["x"], wl["m"], n, steps=steps, warmup=warmup), n


def cpu_best_apply(wl, steps, warmup):
    """The faster of the two ways the reference runs on a host (a short probe
    of each decides), timed over `steps` applies; returns (s, cores, config)."""
    t_omp, n = cpu_reference_apply(wl, 2, 1)
    try:
        t_slab, _ = cpu_slab_apply(wl, 2, 1)
    except Exception:
        t_slab = float("inf")
    if t_slab < t_omp:
        dt, n = cpu_slab_apply(wl, steps, warmup)
        return dt, n, f"{n} processes x 1 thread on z-slabs (MPI-rank layout)"
    dt, n = cpu_reference_apply(wl, steps, warmup)
    return dt, n, f"OpenMP {n} threads"


SOLVE_WORKLOAD = ("Stokes solve, Q2-P1disc 32^3 unit cube, 8 sinkers r=0.1 (eta contrast 1e4, density +1%), "
                  "g=-z, free slip walls/base, free surface top; FGMRES(30) + Schur upper (geometric-mean "
                  "viscosity-scaled mass matrix) + 4-level Galerkin GMG, Chebyshev(3)/Jacobi, rtol 1e-6")


def cpu_solve_sample(m, c, eta, rho, bits, iterations=10):
    """The solver restated on the host cores (oracle/cpu_solver.py: the same
    FGMRES + Schur-upper + Galerkin GMG, with the reference's own AVX operator
    kernels on the fine level), timed over a bounded number of iterations."""
    from oracle.cpu_solver import CpuStokesSolver
    from oracle.oracle import Reference, build
    if not Reference.available():
        build()
    S = CpuStokesSolver(m, c, eta, rho, bits, nlevels=4, threads=os.cpu_count())
    _, _, its, _, dt = S.solve(rtol=1e-6, max_it=iterations)
    return S.setup_s, dt / max(1, its), its


def solve_leg(device, m=32, seed=1, cpu=True):
    """FP64 vs mixed-precision device-resident Stokes solve, each checked
    against an FP64 solve converged to rtol 1e-10; the CPU restatement of the
    same solve timed on a bounded sample of iterations."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.solver import StokesSolver
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(8, seed, 0.1)
    eta = M.sinker_eta(qp, cen, r, 1.0, 1e4)
    rho = M.sinker_density(qp, cen, r, 1.0, 1.01)
    out = {}
    sols = {}
    for name, prec, rtol in (("ref", PREC_F64, 1e-10), ("fp64", PREC_F64, 1e-6), ("mixed", PREC_F32, 1e-6)):
        S = StokesSolver(m, m, m, bits, device=device, nlevels=4, rtol=rtol, max_it=8000, mg_precision=prec,
                         schur_eta=SCHUR_ETA_GEOMEAN)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u, p, st = S.solve(raise_on_noconv=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        sols[name] = (u.cpu().numpy(), p.cpu().numpy())
        out[name] = {"s": dt, "iterations": st["iterations"], "converged": bool(st["converged"]),
                     "rel_residual": st["rfinal"] / st["r0"], "setup_s": st["setup_ms"] * 1e-3}
        S.destroy()
    ur, pr = sols["ref"]
    for name in ("fp64", "mixed"):
        u, p = sols[name]
        out[name]["u_err"] = float(np.linalg.norm(u - ur) / np.linalg.norm(ur))
        out[name]["p_err"] = float(np.linalg.norm(p - pr) / np.linalg.norm(pr))
    (u64, p64), (u32, p32) = sols["fp64"], sols["mixed"]
    cpu_solve = None
    if cpu:
        try:
            setup_s, s_it, its = cpu_solve_sample(m, c, eta, rho, bits)
            est = setup_s + s_it * out["fp64"]["iterations"]
            cpu_solve = {"kind": "port", "cores": os.cpu_count(), "setup_s": setup_s, "s_per_iteration": s_it,
                         "iterations_sampled": its, "est_solve_s": est,
                         "est_speedup_gpu_fp64": est / (out["fp64"]["s"] + out["fp64"]["setup_s"]),
                         "sample": f"setup plus {its} FGMRES iterations of the solver restated on the host "
                                   "(oracle/cpu_solver.py; fine-level operators are the reference's AVX kernels, "
                                   "OpenMP), extrapolated to the FP64 GPU solve's iteration count"}
        except Exception as exc:  # reported, not required
            cpu_solve = {"kind": "port", "sample": f"failed: {exc}"}
    return {"workload": SOLVE_WORKLOAD, "unit": "s", "fp64_s": out["fp64"]["s"], "mixed_s": out["mixed"]["s"],
            "speedup_mixed_vs_fp64": out["fp64"]["s"] / out["mixed"]["s"], "fp64": out["fp64"], "mixed": out["mixed"],
            "u_diff_mixed_vs_fp64": float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64)),
            "p_diff_mixed_vs_fp64": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64)),
            "oracle_solve": out["ref"], "cpu_solve": cpu_solve}


SOLVE_C4_WORKLOAD = ("Stokes solve, Q2-P1disc 96^3 deformed mesh (interior nodes +-0.2h, Jacobians per Gauss point), "
                     "per-element log-normal eta with sigma 1 decade (corr 0.1), 8 sinkers of density +1%, g=-z, "
                     "free slip walls/base, free surface top; FGMRES(30) + Schur upper (geometric mean) + 5-level "
                     "Galerkin GMG, Chebyshev(3)/Jacobi, rtol 1e-6")


SOLVE_C3_WORKLOAD = ("Stokes solve, Q2-P1disc {m}^3 unit cube, layered eta (6 layers, log10 eta in [-3,3], 16 "
                     "inclusions), 8 sinkers of density +1%, g=-z, free slip walls/base, free surface top; "
                     "FGMRES({restart}) + Schur upper (geometric mean) + 5-level Galerkin GMG, Chebyshev(3)/Jacobi, "
                     "rtol 1e-6, at most {max_it} iterations")


def solve_c3_leg(device, m=64, seed=4, max_it=3000, restart=120):
    """FP64 and mixed-precision solves of the layered 64^3 field (eta over six
    decades), each bounded to max_it outer iterations: this preconditioner
    family converges slowly on it (the CPU restatement too; FGMRES(120)
    reaches about 1e-3 in 3,000 iterations where FGMRES(30) stalls near 0.9),
    so the leg records the residual reached and the time per iteration of
    both precisions."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.solver import StokesSolver
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    eta = M.layered_eta(qp, seed=seed)
    cen, r = M.random_sinkers(8, 1, 0.1)
    rho = M.sinker_density(qp, cen, r, 1.0, 1.01)
    out, sols = {}, {}
    for name, prec in (("fp64", PREC_F64), ("mixed", PREC_F32)):
        S = StokesSolver(m, m, m, bits, device=device, nlevels=5, rtol=1e-6, max_it=max_it, mg_precision=prec,
                         schur_eta=SCHUR_ETA_GEOMEAN, restart=restart)
        S.setup(c, eta)
        S.set_rhs_body_force(rho)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u, p, st = S.solve(raise_on_noconv=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        sols[name] = (u.cpu().numpy(), p.cpu().numpy())
        out[name] = {"s": dt, "iterations": st["iterations"], "ms_per_iteration": 1e3 * dt / max(1, st["iterations"]),
                     "converged": bool(st["converged"]), "rel_residual": st["rfinal"] / st["r0"],
                     "setup_s": st["setup_ms"] * 1e-3}
        S.destroy()
        del S, u, p
        torch.cuda.empty_cache()
    (u64, p64), (u32, p32) = sols["fp64"], sols["mixed"]
    return {"workload": SOLVE_C3_WORKLOAD.format(m=m, max_it=max_it, restart=restart), "unit": "s", "fp64": out["fp64"],
            "mixed": out["mixed"],
            "ms_per_iteration_ratio_fp64_vs_mixed": out["fp64"]["ms_per_iteration"] / out["mixed"]["ms_per_iteration"],
            "u_diff_mixed_vs_fp64": float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64)),
            "p_diff_mixed_vs_fp64": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))}


def solve_c4_leg(device, coords, m=96, seed=4):
    """FP64 vs mixed-precision solve on the deformed 96^3 mesh of the apply
    benchmark.  The apply's sigma = 2 decades field spans 12 decades of eta,
    where this preconditioner family stagnates (the CPU restatement too), so
    the solve takes the same construction with sigma = 1 decade."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.solver import StokesSolver
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    eta = M.lognormal_grf_eta(m, m, m, seed=seed, sigma_decades=1.0, corr_len=0.1)
    qp = M.qp_coords(coords, m, m, m)
    cen, r = M.random_sinkers(8, 1, 0.1)
    rho = M.sinker_density(qp, cen, r, 1.0, 1.01)
    out, sols = {}, {}
    for name, prec in (("fp64", PREC_F64), ("mixed", PREC_F32)):
        S = StokesSolver(m, m, m, bits, device=device, nlevels=5, rtol=1e-6, max_it=2000, mg_precision=prec,
                         schur_eta=SCHUR_ETA_GEOMEAN)
        S.setup(coords, eta)
        S.set_rhs_body_force(rho)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u, p, st = S.solve(raise_on_noconv=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        sols[name] = (u.cpu().numpy(), p.cpu().numpy())
        out[name] = {"s": dt, "iterations": st["iterations"], "converged": bool(st["converged"]),
                     "rel_residual": st["rfinal"] / st["r0"], "setup_s": st["setup_ms"] * 1e-3}
        S.destroy()
        del S, u, p
        torch.cuda.empty_cache()
    (u64, p64), (u32, p32) = sols["fp64"], sols["mixed"]
    return {"workload": SOLVE_C4_WORKLOAD, "unit": "s", "fp64_s": out["fp64"]["s"], "mixed_s": out["mixed"]["s"],
            "speedup_mixed_vs_fp64": out["fp64"]["s"] / out["mixed"]["s"], "fp64": out["fp64"], "mixed": out["mixed"],
            "u_diff_mixed_vs_fp64": float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64)),
            "p_diff_mixed_vs_fp64": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))}


def lattice_markers(m, per_dir=2, seed=5):
    """per_dir^3 markers per element of an m^3 mesh, element-major (the
    reference's lattice layout of new markers), local coordinates jittered by
    +-0.25 around the lattice sites, log10 eta uniform in [-3, 3], rho ~ 1."""
    rng = np.random.default_rng(seed)
    nel, k = m ** 3, per_dir ** 3
    s = (np.arange(per_dir) + 0.5) * (2.0 / per_dir) - 1.0
    site = np.stack(np.meshgrid(s, s, s, indexing="ij")[::-1], axis=-1).reshape(-1, 3)
    xi = np.clip(np.tile(site, (nel, 1)) + rng.uniform(-0.25, 0.25, size=(nel * k, 3)), -1.0, 1.0)
    wil = np.repeat(np.arange(nel, dtype=np.int32), k)
    return wil, xi, 10.0 ** rng.uniform(-3.0, 3.0, size=nel * k), rng.uniform(0.99, 1.01, size=nel * k)


def markers_leg(device, m=96, per_dir=2, reps=10, cpu_m=48):
    """Material points onto Gauss points (p3d_marker_project) for the P0
    geometric and Q1 projections on an m^3 mesh, device-timed with CUDA
    events; beside it the reference's own compiled projection on a bounded
    cpu_m^3 sample, one host thread."""
    import torch

    from ptatin3d_b200.markers import PROJ_P0_GEOMETRIC, PROJ_Q1, update_gauss_properties
    wil, xi, eta, rho = lattice_markers(m, per_dir)
    n = wil.size
    dev = torch.device("cuda", device)
    w, x = torch.from_numpy(wil).to(dev), torch.from_numpy(xi).to(dev)
    e, r = torch.from_numpy(eta).to(dev), torch.from_numpy(rho).to(dev)
    eq = torch.empty(m ** 3, 27, dtype=torch.float64, device=dev)
    rq = torch.empty_like(eq)
    out = {"workload": f"{n} markers ({per_dir}^3 per element, element-major) on a {m}^3 mesh", "markers": n}
    st = torch.cuda.current_stream()
    for name, t in (("p0_geometric", PROJ_P0_GEOMETRIC), ("q1", PROJ_Q1)):
        for _ in range(3):
            update_gauss_properties((m, m, m), t, w, x, e, r, eq, rq)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for _ in range(reps):
            update_gauss_properties((m, m, m), t, w, x, e, r, eq, rq)
        t1.record(st)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / reps
        out[name] = {"ms": ms, "Gmarkers/s": n / (ms * 1e-3) / 1e9}
    try:
        from oracle.oracle import Reference, build
        if not Reference.available():
            build()
        from ptatin3d_b200 import mesh as M
        cw, cx, ce, cr = lattice_markers(cpu_m, per_dir)
        R = Reference()
        R.setup((cpu_m,) * 3, M.uniform_coords(cpu_m, cpu_m, cpu_m), np.ones(27 * cpu_m ** 3))
        cpu = {"kind": "reference", "cores": 1,
               "sample": f"the reference's compiled projection, {cw.size} markers on a {cpu_m}^3 mesh, 1 thread"}
        for name, t in (("p0_geometric", 20), ("q1", 1)):
            t0 = time.perf_counter()
            R.marker_project(t, cw, cx, ce, cr)
            cpu[name] = {"s": time.perf_counter() - t0}
            cpu[name]["Gmarkers/s"] = cw.size / cpu[name]["s"] / 1e9
        out["cpu_baseline"] = cpu
    except Exception as exc:  # reported, not required
        out["cpu_baseline"] = {"failed": str(exc)}
    return out


SERVE_SIZES = (8, 12, 16, 24, 32, 48)


def serving_stream(n, seed=7, rate_per_s=200.0):
    """Independent sinker solves: m^3 elements, m uniform in SERVE_SIZES, 1-12
    sinkers of radius 0.1, viscosity contrast log-uniform in [1e2, 1e5],
    density +1 %, Poisson arrivals."""
    from ptatin3d_b200 import mesh as M
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        m = int(rng.choice(SERVE_SIZES))
        nsph = int(rng.integers(1, 13))
        contrast = float(10.0 ** rng.uniform(2.0, 5.0))
        c = M.uniform_coords(m, m, m)
        qp = M.qp_coords(c, m, m, m)
        cen = rng.uniform(0.0, 1.0, size=(nsph, 3))
        out.append(dict(m=m, coords=c, eta=M.sinker_eta(qp, cen, 0.1, 1.0, contrast),
                        rho=M.sinker_density(qp, cen, 0.1, 1.0, 1.01), contrast=contrast, nsph=nsph))
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))
    return out, arrivals - arrivals[0]


def serve_leg(device, n, max_active=8, group_max=8, group_elements=16384):
    """Served stream (mixed precision, rtol 1e-6) against the same solves run
    one after another with the plain FP64 solver."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.serving import StokesServer
    from ptatin3d_b200.solver import StokesSolver, max_levels
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    reqs, arrivals = serving_stream(n)
    opts = dict(rtol=1e-6, max_it=1000, schur_eta=SCHUR_ETA_GEOMEAN)
    # served: continuous admission, concurrent solves
    S = StokesServer(device=device, hbm_budget=64 << 30, max_active=max_active, group_max=group_max,
                     group_elements=group_elements)
    for r in reqs[:6]:  # warm the pool shapes (setup of each shape once)
        S.submit((r["m"],) * 3, bits, r["coords"], r["eta"], r["rho"], nlevels=max_levels(r["m"]),
                 mg_precision=PREC_F32, **opts)
    S.wait_all()
    done, i = [], 0
    t0 = time.perf_counter()
    while len(done) < n:
        now = time.perf_counter() - t0
        while i < n and arrivals[i] <= now:
            r = reqs[i]
            S.submit((r["m"],) * 3, bits, r["coords"], r["eta"], r["rho"], tag=i, nlevels=max_levels(r["m"]),
                     mg_precision=PREC_F32, **opts)
            i += 1
        done += S.poll(timeout_ms=1)
    served_s = time.perf_counter() - t0
    st = S.stats()
    S.close()
    lat = np.array([d["latency_ms"] for d in done])
    lat_ok = np.array([d["latency_ms"] for d in done if d["ok"]] or [float("nan")])
    n_ok = int(sum(d["ok"] for d in done))
    # sequential plain FP64 solves (solvers reused per mesh size), inputs from and results to the host
    pool = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq_ok = 0
    for r in reqs:
        m = r["m"]
        if m not in pool:
            pool[m] = StokesSolver(m, m, m, bits, device=device, nlevels=max_levels(m), mg_precision=PREC_F64, **opts)
        D = pool[m]
        D.setup(r["coords"], r["eta"])
        D.set_rhs_body_force(r["rho"])
        u, p, stt = D.solve(raise_on_noconv=False)
        u.cpu(), p.cpu()
        seq_ok += int(stt["converged"])
    torch.cuda.synchronize()
    seq_s = time.perf_counter() - t0
    for D in pool.values():
        D.destroy()
    return {"workload": f"{n} independent Stokes solves, m^3 elements with m uniform in {list(SERVE_SIZES)}, 1-12 "
                        "sinkers r=0.1, eta contrast log-uniform [1e2,1e5], Poisson arrivals 200/s; mixed precision, "
                        "rtol 1e-6, max 1000 FGMRES iterations",
            "requests": n, "max_active": max_active, "group_max": group_max, "group_elements": group_elements,
            "converged": n_ok,
            "converged_solves_per_s": n_ok / served_s,
            "p50_latency_ms_converged": float(np.percentile(lat_ok, 50)),
            "p99_latency_ms_converged": float(np.percentile(lat_ok, 99)),
            "all_requests": {"solves_per_s": n / served_s, "p50_latency_ms": float(np.percentile(lat, 50)),
                             "p99_latency_ms": float(np.percentile(lat, 99))},
            "sequential_fp64_converged_solves_per_s": seq_ok / seq_s, "sequential_fp64_converged": seq_ok,
            "sequential_fp64_solves_per_s": n / seq_s,
            "speedup_vs_sequential_fp64": seq_s / served_s,
            "converged_speedup_vs_sequential_fp64": (n_ok / served_s) / (seq_ok / seq_s) if seq_ok else None,
            "peak_device_bytes": st["peak_device_bytes"], "solvers_created": st["solvers_created"],
            "solvers_reused": st["solvers_reused"], "grouped_requests": st["grouped"], "groups": st["groups"]}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = workload(args.size, kind=args.workload)
    dt, n, how = cpu_best_apply(wl, args.steps, args.warmup)
    ndof = wl["x"].size
    v = ndof / dt / 1e9
    line = {"metric": metric_name(wl["m"], wl["kind"]), "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(wl["m"], wl["kind"]), "elements": wl["m"] ** 3, "dofs": ndof},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": n, "kind": "reference",
                             "sample": f"{args.steps} full {wl['m']}^3 applies of MFStokesWrapper_A11_AVX ({how})"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import ctypes as C

    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, launch_count
    from ptatin3d_b200._lib import BC_MATMULT, check, lib
    from ptatin3d_b200.operators import MatA11MF, mesh_desc_whole

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    if world > 1:
        return run_slabs(args, rank, world, local)
    if args.slabs:  # the multi-GPU code path on one rank (no neighbour exchange)
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:29531", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120))
        return run_slabs(args, 0, 1, local)
    wl = workload(args.size, kind=args.workload)
    m = wl["m"]
    ndof = wl["x"].size
    desc = mesh_desc_whole(m, m, m, wl["bits"])
    op = MatA11MF(desc, PREC_F64, device=local)
    op.set_coefficients(wl["coords"], wl["eta"])
    L = lib()
    check(L.p3d_op_set_bc_mode(op.h, BC_MATMULT))
    x = torch.tensor(wl["x"], dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    xp, yp = C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())

    def step():  # MatMult_MFStokes_A11: y = A11 x
        check(L.p3d_a11_mult(op.h, xp, yp, sp))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    n0 = launch_count()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for e0, e1 in evs:
            e0.record(stream)
            step()
            e1.record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    launches = launch_count() - n0
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    step_ms = reduce_max(total_ms / args.steps, world)
    value = world * ndof / (step_ms * 1e-3) / 1e9

    # FP32 operator on the same mesh (the mixed-precision smoother's apply)
    op32 = MatA11MF(desc, PREC_F32, device=local)
    op32.set_coefficients(wl["coords"], wl["eta"])
    check(L.p3d_op_set_bc_mode(op32.h, BC_MATMULT))
    x32, y32 = x.float(), torch.zeros(ndof, dtype=torch.float32, device="cuda")
    for _ in range(3):
        check(L.p3d_a11_mult(op32.h, C.c_void_p(x32.data_ptr()), C.c_void_p(y32.data_ptr()), sp))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        check(L.p3d_a11_mult(op32.h, C.c_void_p(x32.data_ptr()), C.c_void_p(y32.data_ptr()), sp))
    e1.record(stream)
    torch.cuda.synchronize()
    f32_ms = e0.elapsed_time(e1) / args.steps
    f32_err = float((y32.double() - y).norm() / y.norm())  # y = A x from the last FP64 step
    del op32, x32, y32

    # end to end through the reference-facing host-buffer call (x in, y out each step)
    if args.no_e2e:
        args.steps_e2e = 0
    xh = torch.tensor(wl["x"], dtype=torch.float64).pin_memory()
    yh = torch.zeros(ndof, dtype=torch.float64).pin_memory()
    xhp, yhp = C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr())
    for _ in range(2):
        check(L.p3d_a11_apply_host(op.h, xhp, yhp))
    barrier(world)
    t0 = time.perf_counter()
    ne2e = max(3, args.steps // 2) if not args.no_e2e else 1
    for _ in range(ne2e):
        check(L.p3d_a11_apply_host(op.h, xhp, yhp))
    e2e_s = reduce_max((time.perf_counter() - t0) / ne2e, world)
    e2e_value = world * ndof / e2e_s / 1e9
    # the same call on pageable host arrays, as a PETSc MatShell callback hands
    # over its local vectors (the copies go through the driver's staging)
    xpg = np.ascontiguousarray(wl["x"], dtype=np.float64)
    ypg = np.zeros(ndof)
    xpp, ypp = C.c_void_p(xpg.ctypes.data), C.c_void_p(ypg.ctypes.data)
    check(L.p3d_a11_apply_host(op.h, xpp, ypp))
    t0 = time.perf_counter()
    npg = max(3, ne2e // 4)
    for _ in range(npg):
        check(L.p3d_a11_apply_host(op.h, xpp, ypp))
    pg_value = world * ndof / reduce_max((time.perf_counter() - t0) / npg, world) / 1e9
    # and with the operator page-locking those arrays on first use (kept across calls)
    check(L.p3d_op_set_host_register(op.h, 1))
    check(L.p3d_a11_apply_host(op.h, xpp, ypp))  # registers
    t0 = time.perf_counter()
    for _ in range(ne2e):
        check(L.p3d_a11_apply_host(op.h, xpp, ypp))
    pgr_value = world * ndof / reduce_max((time.perf_counter() - t0) / ne2e, world) / 1e9
    check(L.p3d_op_set_host_register(op.h, 0))
    # the pipelined host-buffer result is the device MatMult's
    check(L.p3d_a11_mult(op.h, xp, yp, sp))
    torch.cuda.synchronize()
    e2e_diff = float((yh.to("cuda") - y).norm() / y.norm())

    peak, peak_kind = load_peaks()
    ab = algorithmic_bytes(m)
    achieved = ab / (kern_ms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.txt")  # ncu dram__bytes_read+write per launch
    if os.path.exists(tf) and m == 96 and args.workload == "deformed":
        for ln in open(tf):
            f = ln.split()
            if len(f) == 2 and f[0] == "a11_f64_general_96":
                traffic = float(f[1])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            sub = dict(wl)
            dt, n = cpu_reference_apply(sub, steps=20, warmup=2)
            dt1, _ = cpu_reference_apply(sub, steps=1, warmup=0, threads=1)
            try:
                dts, ns = cpu_slab_apply(sub, steps=20, warmup=2)
            except Exception:
                dts, ns = float("inf"), 0
            best = min(dt, dts)
            cpu = {"value": ndof / best / 1e9, "unit": UNIT, "cores": ns if dts < dt else n, "kind": "reference",
                   "sample": f"best of two layouts of the reference MFStokesWrapper_A11_AVX (oracle/_ref), 20 full "
                             f"{m}^3 applies each after 2 warm-up applies: "
                             + ("z-slabs, one process per core" if dts < dt else f"OpenMP {n} threads"),
                   "openmp": {"value": ndof / dt / 1e9, "unit": UNIT, "threads": n},
                   "slabs": {"value": ndof / dts / 1e9 if dts < float("inf") else None, "unit": UNIT, "processes": ns,
                             "sample": "one z-slab per process, 1 thread each, started at a barrier; time of the "
                                       "slowest slab; the shared-plane sums are not timed"},
                   "single_thread": {"value": ndof / dt1 / 1e9, "unit": UNIT, "sample": f"1 full {m}^3 apply, 1 thread"}}
        except Exception as exc:  # the baseline is reported, not required
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {exc}"}

    solve = None
    if rank == 0 and not args.no_solve:
        solve = solve_leg(local, cpu=not args.no_cpu)
        if m == 96 and args.workload == "deformed":
            try:
                solve["deformed_96"] = solve_c4_leg(local, wl["coords"])
            except Exception as exc:  # reported, not required
                solve["deformed_96"] = {"failed": str(exc)}
            try:
                solve["layered_64"] = solve_c3_leg(local)
            except Exception as exc:  # reported, not required
                solve["layered_64"] = {"failed": str(exc)}
    serving = None
    if rank == 0 and args.serve_requests > 0:
        serving = serve_leg(local, args.serve_requests, group_max=args.serve_group_max,
                            group_elements=args.serve_group_elements)
    grouped = None
    if rank == 0 and args.serve_requests > 0:
        try:
            grouped = grouped_leg(local)
        except Exception as exc:  # reported, not required
            grouped = {"failed": str(exc)}
    markers = None
    if rank == 0 and not args.no_markers:
        try:
            markers = markers_leg(local, m)
        except Exception as exc:  # reported, not required
            markers = {"failed": str(exc)}

    if rank == 0:
        line = {"metric": metric_name(m, wl["kind"]), "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload_name(m, wl["kind"]),
                           "elements": m ** 3, "dofs": ndof, "geometry_path": "general" if op.geometry_mode == 1 else "affine",
                           "l2": "inputs > L2 (709 MB/apply), no flush", "parallelism": f"replicas x{world}"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "algorithmic_bytes": ab, "kernel_ms": kern_ms},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * ndof, "d2h_bytes_per_step": 8 * ndof,
                        "rel_diff_vs_device": e2e_diff, "host_buffers": "pinned",
                        "pageable": {"value": pg_value, "unit": UNIT, "steps": npg,
                                     "sample": "the same call on pageable numpy arrays"},
                        "pageable_registered": {"value": pgr_value, "unit": UNIT, "steps": ne2e,
                                                "sample": "pageable numpy arrays page-locked by the operator on "
                                                          "first use (p3d_op_set_host_register), kept across calls"}},
                "gpu_launches": launches,
                "clocks": clk.summary(),
                "fp32_apply": {"ms": f32_ms, "GDoF/s": ndof / (f32_ms * 1e-3) / 1e9,
                               "hbm_frac": algorithmic_bytes(m, 4) / (f32_ms * 1e-3) / 1e9 / peak,
                               "rel_err_vs_fp64": f32_err},
                "fp64_alu": {"flop_per_element": REF_FLOPS_PER_EL,
                             "TFLOP/s": REF_FLOPS_PER_EL * m ** 3 / (kern_ms * 1e-3) / 1e12},
                "solve": solve,
                "serving": serving,
                "grouped_solves": grouped,
                "markers": markers}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_slabs(args, rank, world, local):
    """N GPUs: one mesh of m x m x (m*N) elements cut into z-slabs of m^3
    elements, one per rank (weak scaling).  A step is one A11 MatMult of the
    whole mesh: every rank applies its slab, then the node plane shared with
    each neighbour is exchanged point-to-point over NCCL and added
    (DMLocalToGlobal(ADD) of a 1-D decomposition)."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from ptatin3d_b200 import PREC_F64, launch_count
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200._lib import BC_MATMULT, check, lib
    from ptatin3d_b200.slabs import SlabExchange, device_slab_operator, slab_range
    m = args.size
    mzg = m * world
    z0, z1 = slab_range(mzg, rank, world)
    coords = M.slab_coords(m, m, mzg, z0, z1, frac=0.2, seed=4)
    eta = M.lognormal_grf_eta(m, m, z1 - z0, seed=4 + 1000 * rank, sigma_decades=2.0, corr_len=0.1)
    op = device_slab_operator(m, m, mzg, M.FREE_SLIP, coords, eta, rank, world, PREC_F64, local)
    L = lib()
    check(L.p3d_op_set_bc_mode(op.h, BC_MATMULT))
    ex = SlabExchange(m, m, mzg, M.FREE_SLIP, rank, world, device=torch.device("cuda", local))
    rng = np.random.default_rng(100 + rank)
    x = torch.tensor(rng.uniform(-1.0, 1.0, size=ex.n_local), dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    xp, yp = C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())

    def step():  # slab MatMult, then the shared planes' partial sums
        check(L.p3d_a11_mult(op.h, xp, yp, sp))
        ex.add_shared(x, y)

    dist.barrier()
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    n0 = launch_count()
    with ClockSampler(local) as clk:
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
    launches = launch_count() - n0
    step_ms = reduce_max(t0.elapsed_time(t1) / args.steps, world)
    ndof = 3 * (2 * m + 1) ** 2 * (2 * mzg + 1)  # unique dofs of the whole mesh
    value = ndof / (step_ms * 1e-3) / 1e9
    # end to end: the slab's x from pinned host memory in, y out, every step
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    ne = max(3, args.steps // 10)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ne):
        x.copy_(xh, non_blocking=True)
        step()
        yh.copy_(y, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1) / ne, world)
    peak, peak_kind = load_peaks()
    ab = world * algorithmic_bytes(m)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"A11 MatMult, Q2 {m}x{m}x{mzg} deformed mesh (interior nodes +-0.2h), "
                                       "log-normal eta, free-slip walls; z-slabs of m^3 elements per GPU with a "
                                       "shared-plane exchange over NCCL every step",
                           "elements": m * m * mzg, "dofs": ndof, "parallelism": f"z-slabs x{world}",
                           "l2": "inputs > L2 per GPU, no flush"},
                "roofline": {"bound": "hbm", "achieved": ab / world / (step_ms * 1e-3) / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": ab / world / (step_ms * 1e-3) / 1e9 / peak, "traffic": None,
                             "peak_kind": peak_kind, "note": "per GPU, step time including the exchange"},
                "cpu_baseline": None,
                "e2e": {"value": ndof / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
                        "h2d_bytes_per_step": 8 * ex.n_local * world, "d2h_bytes_per_step": 8 * ex.n_local * world},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    del op
    dist.destroy_process_group()
    return 0


def profile_solve(spec):
    """One short solve for profiling its kernel mix: spec =
    "m,iterations,precision[,deformed]" (precision 64 or 32).  Default: the C2
    construction (unit cube, 8 sinkers of radius 0.1, viscosity contrast 1e4,
    density +1 %, free slip walls and base, free surface top, 4 Galerkin
    levels); "deformed": the deformed-mesh solve of the apply benchmark
    (interior nodes +-0.2h, log-normal eta of sigma 1 decade, 5 levels).
    Chebyshev(3)/Jacobi, geometric-mean Schur weighting; stops after
    `iterations` FGMRES iterations.  Prints one line, no JSON (not a
    benchmark number)."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.solver import StokesSolver, max_levels
    parts = spec.split(",")
    m, its, prec = (int(v) for v in parts[:3])
    deformed = len(parts) > 3 and parts[3] == "deformed"
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    c = M.uniform_coords(m, m, m)
    if deformed:
        c = M.perturb_interior(c, m, m, m, frac=0.2, seed=4)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(8, 1, 0.1)
    eta = (M.lognormal_grf_eta(m, m, m, seed=4, sigma_decades=1.0, corr_len=0.1) if deformed
           else M.sinker_eta(qp, cen, r, 1.0, 1e4))
    S = StokesSolver(m, m, m, bits, nlevels=min(5 if deformed else 4, max_levels(m)), rtol=1e-12, max_it=its,
                     mg_precision=PREC_F32 if prec == 32 else PREC_F64, schur_eta=SCHUR_ETA_GEOMEAN)
    S.setup(c, eta)
    S.set_rhs_body_force(M.sinker_density(qp, cen, r, 1.0, 1.01))
    u, p, st = S.solve(raise_on_noconv=False)
    torch.cuda.synchronize()
    print(f"{st['iterations']} iterations, |r|/|r0| = {st['rfinal'] / st['r0']:.3e}, "
          f"setup {st['setup_ms']:.1f} ms, solve {st['solve_ms']:.1f} ms")
    S.destroy()
    return 0


def grouped_solves(m, K, its, prec, device=0):
    """K solves of one shape, first one after another and then as one grouped
    solve (p3d_solver_solve_grouped).  Each member is a unit cube with its own
    4 sinkers of radius 0.1 (viscosity contrast 1e3, density +1 %), free slip
    walls and base, free surface top, Chebyshev(3)/Jacobi, Galerkin levels
    down to 2^3 elements or fewer, geometric-mean Schur weighting; every solve
    stops after `its` FGMRES iterations.  Returns (one-after-another ms,
    grouped ms, member iterations)."""
    import torch

    from ptatin3d_b200 import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
    from ptatin3d_b200 import mesh as M
    from ptatin3d_b200.solver import StokesSolver, max_levels, solve_grouped
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    solvers = []
    for s in range(K):
        cen, r = M.random_sinkers(4, s + 1, 0.1)
        S = StokesSolver(m, m, m, bits, device=device, nlevels=max_levels(m), rtol=1e-14, max_it=its,
                         mg_precision=PREC_F32 if prec == 32 else PREC_F64, schur_eta=SCHUR_ETA_GEOMEAN)
        S.setup(c, M.sinker_eta(qp, cen, r, 1.0, 1e3))
        S.set_rhs_body_force(M.sinker_density(qp, cen, r, 1.0, 1.01))
        solvers.append(S)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for S in solvers:
        S.solve(raise_on_noconv=False)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = solve_grouped(solvers)
    torch.cuda.synchronize()
    t_grp = time.perf_counter() - t0
    n_its = sum(r[2]["iterations"] for r in res)
    for S in solvers:
        S.destroy()
    return t_seq * 1e3, t_grp * 1e3, n_its


def profile_group(spec):
    """grouped_solves for profiling their launches: spec = "m,K,iterations,
    precision".  Prints the wall times, no JSON (not a benchmark number)."""
    m, K, its, prec = (int(v) for v in spec.split(","))
    t_seq, t_grp, n_its = grouped_solves(m, K, its, prec)
    print(f"{K} solves of {m}^3, {its} iterations each: one after another {t_seq:.1f} ms, grouped "
          f"{t_grp:.1f} ms ({n_its} member iterations, {t_grp / n_its:.3f} ms each)")
    return 0


def grouped_leg(device):
    """Shared launches: 8 same-shape small solves (mixed precision, 30 FGMRES
    iterations each) one after another and as one grouped solve."""
    out = {"workload": "8 same-shape Stokes solves (unit cube, 4 sinkers each, contrast 1e3), mixed precision, "
                       "30 FGMRES iterations each: one after another vs p3d_solver_solve_grouped"}
    for m in (8, 16):
        grouped_solves(m, 8, 3, 32, device)  # warm-up (graphs, pools)
        t_seq, t_grp, n_its = grouped_solves(m, 8, 30, 32, device)
        out[f"m{m}"] = {"one_after_another_ms": t_seq, "grouped_ms": t_grp, "member_iterations": n_its,
                        "speedup": t_seq / t_grp}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-solve", action="store_true", help="skip the FP64 vs mixed-precision Stokes solve leg")
    ap.add_argument("--serve-requests", type=int, default=256, help="requests of the served-stream leg (0: skip)")
    ap.add_argument("--serve-group-max", type=int, default=8,
                    help="queued same-shape requests the server solves as one group (1: no grouping)")
    ap.add_argument("--serve-group-elements", type=int, default=16384,
                    help="largest mesh (elements) the server solves in groups")
    ap.add_argument("--no-markers", action="store_true", help="skip the marker-projection leg")
    ap.add_argument("--slabs", action="store_true", help="run the multi-GPU z-slab path on a single rank")
    ap.add_argument("--size", type=int, default=96, help="elements per direction")
    ap.add_argument("--workload", default="deformed", choices=["deformed", "layered"])
    ap.add_argument("--profile-solve", default=None, metavar="M,ITS,PREC",
                    help="run one short solve for profiling its launches, print one line, no benchmark")
    ap.add_argument("--profile-group", default=None, metavar="M,K,ITS,PREC",
                    help="run K same-shape solves one after another, then grouped, for profiling; no benchmark")
    args = ap.parse_args()
    if args.profile_solve:
        return profile_solve(args.profile_solve)
    if args.profile_group:
        return profile_group(args.profile_group)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
