"""Benchmark: Darcy head solves/s at 256^3 (||b - A h|| / ||b|| <= 1e-10) + face velocity.

Workload (default): 256 x 256 x 256 cells, lnK Gaussian with variance 4, exponential
covariance, correlation length 8 cells, randomization method with 1000 modes (seeded
synthetic field, no dataset), h = 1 at x = 0, h = 0 at x = L, no-flow elsewhere.  One step
= set-up from K (coarsening, face coefficients, RHS) + PCG to 1e-10 + face velocities, K
resident in HBM.  Every array is larger than L2 (126 MB), so no flush is needed.

Arms:
  default           this library (mixed precision: FP32 V-cycle in flexible FP64 PCG), with
                    the plain FP64 CCMG-PCG of this library measured beside it;
  --impl reference  the reference's own solve_head (PCG_MG) + compute_velocity_from_head,
                    compiled from its sources into oracle/_ref, on the same K and tolerance.
Multi-GPU (torchrun): independent replicas, one realisation per rank, no collective on the
data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
T0 = time.perf_counter()


def note(msg):
    """Progress on stderr (stdout carries only the JSON line)."""
    print(f"[bench {time.perf_counter() - T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def host_cores():
    """Cores this process may use: the CPU affinity mask, capped by a cgroup CPU quota (a
    container can see every core of the host but be allowed only a few; OpenMP with one thread
    per visible core then oversubscribes the allowed ones)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    quota = None
    try:
        q, per = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if q != "max":
            quota = int(q) / int(per)
    except (OSError, ValueError):
        try:
            q = int(open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read())
            per = int(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
            if q > 0 and per > 0:
                quota = q / per
        except (OSError, ValueError):
            pass
    if quota is not None:
        n = min(n, max(1, int(quota)))
    return max(1, n)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            self.f.flush()
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        finally:
            os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_K(M, n, sigma2, lam, seed, device):
    """lam: one correlation length, or (lambda_x, lambda_y, lambda_z)."""
    import torch
    g = M.Grid3D(n, n, n, 1.0)
    lams = tuple(lam) if isinstance(lam, (tuple, list)) else (lam, lam, lam)
    with torch.cuda.device(device):
        return M.generate_K_field(g, sigma2, lams, seed=seed, n_modes=1000)


# the workloads: C2 (256^3, the headline), C1 (64^3 parity case), C3 (512^3, anisotropic)
CONFIGS = {"c2": (256, 4.0, 8.0), "c1": (64, 1.0, 4.0), "c3": (512, 1.0, (16.0, 16.0, 4.0))}


def levels_for(n):
    lv, m = 1, n
    while m > 4 and m % 2 == 0:
        m //= 2
        lv += 1
    return lv


USE_GRAPH = 1


# ---- replicas (N > 1): one independent solve per rank, no collective on the data path ----
def replica_seed(base, rank):
    """Each rank solves its own realisation: seed + rank (EnsembleRunner's seed + r)."""
    return base + rank


def max_over_ranks(dist_ctx, ms, device):
    """The job's time is the slowest rank's (the only collective: one scalar all-reduce)."""
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist_ctx.all_reduce(t, op=dist_ctx.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, steps, ms):
    """Whole-job solves/s: every rank ran `steps` solves within the slowest rank's `ms`."""
    return world * steps / (ms / 1e3)


def solver_cfg(M, n, precision, rtol=1e-10):
    return M.HeadSolveConfig(mg_levels=levels_for(n), mg_pre_smooth=2, mg_post_smooth=2,
                             mg_coarse_iters=50, cg_max_iter=500, cg_check_every=1, cg_rtol=rtol,
                             conv_norm=M.CONV_B, precision=precision, use_graph=USE_GRAPH)


def run_steps(M, n, K, precision, steps, warmup, dist_ctx=None, warmstart=None):
    """Times `steps` device-resident steps; returns dict with per-step ms and last result.
    With `warmstart`, every step also runs the network's inference and solves from its guess."""
    import torch
    g = M.Grid3D(n, n, n, 1.0)
    bc = M.BCSpec.darcy_x()
    stream = torch.cuda.current_stream()
    s = M.HeadSolver(g, bc, solver_cfg(M, n, precision), stream=stream.cuda_stream)
    h = torch.empty_like(K)
    x0 = torch.empty_like(K) if warmstart is not None else None
    su, sv, sw = M.velocity_sizes(g)
    U = torch.empty(su, dtype=torch.float64, device=K.device)
    V = torch.empty(sv, dtype=torch.float64, device=K.device)
    W = torch.empty(sw, dtype=torch.float64, device=K.device)

    def step():
        s.set_K(K)
        if warmstart is not None:
            warmstart.predict(g, bc, K, x0)
        r = s.solve(h, x0)
        M.compute_velocity_from_head(U, V, W, h, K, g, bc)
        return r

    res = None
    for _ in range(warmup):
        res = step()
    if dist_ctx is not None:
        dist_ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    iters = []
    for _ in range(steps):
        res = step()
        iters.append(res.num_iterations)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist_ctx is not None:
        dist_ctx.barrier()
    ms = e0.elapsed_time(e1)
    return dict(solver=s, ms_total=ms, res=res, iters=iters, h=h, launches=s.setup_launches + res.kernel_launches + 1)


def e2e_steps(M, n, K_host, precision, steps, warmup):
    """Same metric through the public API with HOST buffers: H2D of K from pinned memory,
    set-up + solve + velocity, D2H of the head, every step.  The copies run on a second
    stream, double-buffered: step i+1's K goes up and step i-1's head comes down while step i
    solves; every copy of every timed step is inside the timed region (the first upload after
    the start event, the last download before the end event)."""
    import torch
    g = M.Grid3D(n, n, n, 1.0)
    bc = M.BCSpec.darcy_x()
    sa = torch.cuda.current_stream()
    sb = torch.cuda.Stream()
    s = M.HeadSolver(g, bc, solver_cfg(M, n, precision), stream=sa.cuda_stream)
    Kd = [torch.empty(K_host.shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    hd = [torch.empty_like(Kd[0]) for _ in range(2)]
    h_host = [torch.empty(K_host.shape, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    su, sv, sw = M.velocity_sizes(g)
    U = torch.empty(su, dtype=torch.float64, device="cuda")
    V = torch.empty(sv, dtype=torch.float64, device="cuda")
    W = torch.empty(sw, dtype=torch.float64, device="cuda")

    def run(nsteps, e0=None, e1=None):
        k_in = [torch.cuda.Event() for _ in range(2)]    # K of buffer j on the device
        used = [torch.cuda.Event() for _ in range(2)]    # step done with K / head buffer j
        h_out = [torch.cuda.Event() for _ in range(2)]   # head of buffer j on the host
        started = [False, False]

        def upload(j):
            with torch.cuda.stream(sb):
                if started[j]:
                    sb.wait_event(used[j])
                Kd[j].copy_(K_host, non_blocking=True)
                k_in[j].record(sb)

        if e0 is not None:
            e0.record(sa)
        sb.wait_stream(sa)
        upload(0)
        for i in range(nsteps):
            j = i & 1
            if i + 1 < nsteps:
                upload(j ^ 1)
            sa.wait_event(k_in[j])
            if started[j]:
                sa.wait_event(h_out[j])  # the head buffer's last download is done
            s.set_K(Kd[j])
            s.solve(hd[j])
            M.compute_velocity_from_head(U, V, W, hd[j], Kd[j], g, bc)
            used[j].record(sa)
            started[j] = True
            with torch.cuda.stream(sb):
                sb.wait_event(used[j])
                h_host[j].copy_(hd[j], non_blocking=True)
                h_out[j].record(sb)
        sa.wait_stream(sb)
        if e1 is not None:
            e1.record(sa)

    run(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    run(steps, e0, e1)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nbytes = K_host.numel() * 8
    s.close()
    return steps / (ms / 1e3), nbytes, nbytes


def warmstart_eval(M, precision, seed):
    """Config C5: the shipped network (trained on 2000 solver-generated pairs at 128^3) as the
    PCG initial guess at 128^3 and 256^3 on held-out fields, against the zero guess and the
    reference's x-linear guess; PCG runs to ||r||/||b|| <= 1e-10 in every case."""
    import numpy as np
    import torch
    ws = M.WarmStart.pretrained()
    bc = M.BCSpec.darcy_x()
    stream = torch.cuda.current_stream()
    cases = []
    for n in (128, 256):
        g = M.Grid3D(n, n, n, 1.0)
        s = M.HeadSolver(g, bc, solver_cfg(M, n, precision), stream=stream.cuda_stream)
        for k, (s2, lam) in enumerate([(1.0, 6.0), (2.5, 8.0), (4.0, 10.0)]):
            note(f"held-out field {n}^3, sigma2 {s2:g}, lambda {lam:g}")
            K = M.generate_K_field(g, s2, (lam, lam, lam), seed=seed + 9_000_000 + 100 * n + k, n_modes=1000)
            s.set_K(K)
            h = torch.empty_like(K)
            x0 = torch.zeros_like(K)
            s.solve(h)  # warm-up of this grid's graph
            r_lin = s.solve(h)
            href = h.clone()
            r_zero = s.solve(h, x0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ws.predict(g, bc, K, x0)
            e0.record(stream)
            ws.predict(g, bc, K, x0)
            e1.record(stream)
            torch.cuda.synchronize()
            t_inf = e0.elapsed_time(e1)
            err_nn = float((x0 - href).norm() / href.norm())
            hl = torch.from_numpy(np.broadcast_to(1.0 - (np.arange(n) + 0.5) / n, (n, n, n)).copy()).to(K.device)
            err_lin = float((hl - href).norm() / href.norm())
            r_nn = s.solve(h, x0)
            coarse = None
            if n >= 256:
                # the network at half resolution: K coarsened to (n/2)^3 (geometric mean), the
                # predicted correction to the linear head interpolated trilinearly to n^3
                nc = n // 2
                gc = M.Grid3D(nc, nc, nc, 2.0)
                Kc = torch.empty(nc ** 3, dtype=torch.float64, device=K.device)
                xc = torch.empty_like(Kc)
                hlc = torch.from_numpy(np.broadcast_to(1.0 - (np.arange(nc) + 0.5) / nc, (nc, nc, nc)).copy()).to(K.device)

                def coarse_guess():
                    M.coarsen_K(gc, K, Kc)
                    ws.predict(M.Grid3D(nc, nc, nc, 1.0), bc, Kc, xc)
                    dc = (xc.view(1, 1, nc, nc, nc) - hlc.view(1, 1, nc, nc, nc)).float()
                    d = torch.nn.functional.interpolate(dc, scale_factor=2, mode="trilinear", align_corners=False)
                    x0.view(-1).copy_(hl.reshape(-1) + d.reshape(-1).double())
                coarse_guess()
                e0.record(stream)
                coarse_guess()
                e1.record(stream)
                torch.cuda.synchronize()
                t_c = e0.elapsed_time(e1)
                err_c = float((x0 - href).norm() / href.norm())
                r_c = s.solve(h, x0)
                coarse = {"iterations": r_c.num_iterations, "guess_rel_error": err_c,
                          "inference_ms": round(t_c, 3), "solve_ms_incl_inference": round(r_c.device_ms + t_c, 3),
                          "true_rel_residual": r_c.true_rel_residual}
            cases.append({"n": n, "sigma2": s2, "lambda": lam,
                          "iterations": {"zero": r_zero.num_iterations, "linear": r_lin.num_iterations,
                                         "learned": r_nn.num_iterations},
                          "solve_ms": {"zero": round(r_zero.device_ms, 3), "linear": round(r_lin.device_ms, 3),
                                       "learned_incl_inference": round(r_nn.device_ms + t_inf, 3)},
                          "inference_ms": round(t_inf, 3),
                          "guess_rel_error": {"zero": 1.0, "linear": err_lin, "learned": err_nn},
                          "true_rel_residual_learned": r_nn.true_rel_residual,
                          "head_rel_diff_learned_vs_linear": float((h - href).abs().max() / href.abs().max()),
                          "learned_at_half_resolution": coarse})
        s.close()
    ws.close()
    return {"network": "3-D U-Net, 4 levels, 16/32/64/64 channels, 3x3x3, BF16 / FP32 accumulate (tcgen05)",
            "training": "2000 solver-generated pairs at 128^3, lnK variance U(0.5, 4), correlation length U(4, 12); "
                        "3 epochs of Adam, minibatch 4 (macroflow3d_b200.warmstart_train)",
            "held_out": "seeds outside the training set", "cases": cases}


ENSEMBLE_EDGES = (64, 96, 128, 160)


ENSEMBLE_TIMEOUT_S = 240


def ensemble_isolated(cmd, timeout_s):
    """The ensemble record from `cmd` (bench.py --ensemble-only) run as a child process with
    its own CUDA context and a time limit, so that the headline record does not depend on it:
    a child that fails or runs out of time gives {"unavailable": why} instead.  The child's
    progress lines are passed on to stderr."""
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"the ensemble run exceeded {timeout_s} s"}
    for ln in (p.stderr or "").splitlines()[-8:]:
        print(ln, file=sys.stderr, flush=True)
    if p.returncode != 0:
        tail = (p.stderr or "").strip().splitlines()
        return {"unavailable": f"the ensemble run exited {p.returncode}: {tail[-1] if tail else ''}"[:300]}
    try:
        return json.loads(p.stdout.strip().splitlines()[-1])["ensemble"]
    except (ValueError, KeyError, IndexError):
        return {"unavailable": "the ensemble run printed no record"}


def ensemble_shapes(seed, count):
    """Grid edges drawn uniformly from ENSEMBLE_EDGES per axis and realisation (uneven sizes)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [tuple(int(e) for e in rng.choice(ENSEMBLE_EDGES, 3)) for _ in range(count)]


def ensemble_steps(M, prec, count, steps, warmup, seed, tune_reps=3):
    """Monte Carlo ensemble: `count` realisations of uneven grids (sigma^2 = 2, lambda = 6, seed
    + r), each step = set-up from K + PCG to ||r||/||b|| <= 1e-10 + face velocity for every
    realisation.  Batched (mf3d_batch_*: one graph for all) against looping single solves
    (one HeadSolver per distinct grid, reused as FlowWorkspace is)."""
    import torch
    shapes = ensemble_shapes(seed, count)
    grids = [M.Grid3D(nx, ny, nz, 1.0) for nx, ny, nz in shapes]
    lv = min(levels_for(e) for sh in shapes for e in sh)
    cfg = M.HeadSolveConfig(mg_levels=max(lv, 6), mg_pre_smooth=2, mg_post_smooth=2, mg_coarse_iters=50,
                            cg_max_iter=500, cg_check_every=1, cg_rtol=1e-10, conv_norm=M.CONV_B,
                            precision=prec, use_graph=USE_GRAPH)
    bc = M.BCSpec.darcy_x()
    stream = torch.cuda.current_stream()
    Ks = [M.generate_K_field(g, 2.0, (6.0, 6.0, 6.0), seed=seed + r, n_modes=1000) for r, g in enumerate(grids)]
    hs = [torch.empty_like(K) for K in Ks]
    vel = [[torch.empty(q, dtype=torch.float64, device="cuda") for q in M.velocity_sizes(g)] for g in grids]
    cells = sum(g.num_cells() for g in grids)

    def velocities():
        for g, h, K, (U, V, W) in zip(grids, hs, Ks, vel):
            M.compute_velocity_from_head(U, V, W, h, K, g, bc)

    def timed(step):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(steps):
            out = step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    # ---- batched ----
    b = M.BatchSolver(grids, bc, cfg, stream=stream.cuda_stream)
    solvers = {}
    try:
        return _ensemble_arms(M, b, solvers, grids, shapes, bc, cfg, Ks, hs, velocities, timed, cells, count,
                              steps, warmup, tune_reps)
    finally:
        torch.cuda.synchronize()
        b.close()
        for s in solvers.values():
            s.close()


def _ensemble_arms(M, b, solvers, grids, shapes, bc, cfg, Ks, hs, velocities, timed, cells, count, steps, warmup,
                   tune_reps):
    import torch
    stream = torch.cuda.current_stream()
    b.set_K(Ks)
    tuning = b.autotune(tune_reps) if tune_reps > 0 else []
    note(f"ensemble: autotuned {len(tuning)} positions; batched steps")

    def bstep():
        b.set_K(Ks)
        r = b.solve(hs)
        velocities()
        return r

    ms_b, res_b = timed(bstep)
    note("ensemble: looped single solves")
    h_batch = [h.clone() for h in hs[:4]]
    # ---- looping single solves ----
    for g, sh in zip(grids, shapes):
        if sh not in solvers:
            solvers[sh] = M.HeadSolver(g, bc, cfg, stream=stream.cuda_stream)

    def lstep():
        out = []
        for sh, K, h in zip(shapes, Ks, hs):
            s = solvers[sh]
            s.set_K(K)
            out.append(s.solve(h))
        velocities()
        return out

    ms_l, res_l = timed(lstep)
    dh = max(((a - h).abs().max() / h.abs().max()).item() for a, h in zip(h_batch, hs[:4]))
    its_b = [r.num_iterations for r in res_b]
    its_l = [r.num_iterations for r in res_l]
    out = {"workload": f"{count} realisations, edges from {{{','.join(map(str, ENSEMBLE_EDGES))}}} per axis, "
                       "sigma2 2, lambda 6, seed + r, FP32 V-cycle in flexible FP64 PCG to ||r||/||b|| <= 1e-10",
           "cells_total": cells, "distinct_grids": len(solvers),
           "step": "set-up from K + PCG + face velocity, every realisation",
           "batched_solves_per_s": round(count * steps / (ms_b / 1e3), 3),
           "looped_solves_per_s": round(count * steps / (ms_l / 1e3), 3),
           "speedup_batched_vs_looped": round(ms_l / ms_b, 3),
           "batched_cell_solves_per_s": round(cells * steps / (ms_b / 1e3), 1),
           "batched_ms_per_step": round(ms_b / steps, 3), "looped_ms_per_step": round(ms_l / steps, 3),
           "iterations_batched": [min(its_b), max(its_b)], "iterations_looped": [min(its_l), max(its_l)],
           "all_converged": bool(all(r.converged for r in res_b) and all(r.converged for r in res_l)),
           "max_true_rel_residual": max(r.true_rel_residual for r in res_b),
           "head_rel_maxdiff_batched_vs_looped": dh,
           "batched_launches_per_step": res_b[0].kernel_launches,
           "autotune_positions": len(tuning),
           "autotune_gain_ms": round(sum(t["ms_default"] - t["ms_best"] for t in tuning), 4),
           "steps": steps, "warmup": warmup, "device_bytes_batched": b.device_bytes}
    return out


def oracle_rtol(O, K_np, bc):
    """The reference's stopping test is ||r||/||r0|| < rtol; this rtol makes it ||r||/||b|| <= 1e-10."""
    import numpy as np
    b = O.build_rhs(K_np, bc)
    r0 = np.linalg.norm(b - O.apply_A(K_np, O.init_guess(K_np.shape, bc), bc))
    return 1e-10 * np.linalg.norm(b) / r0


def cpu_baseline(K_np, n, budget_s=60.0, reps=3):
    """The oracle (OpenMP restatement of the reference CCMG-PCG) on all host cores: the median
    of `reps` FULL solves (set-up + PCG to ||r||/||b|| <= 1e-10 + one velocity pass) of the
    same workload; fewer when one solve alone takes more than a third of `budget_s`."""
    from oracle import oracle as O
    cores = host_cores()
    O.set_threads(cores)
    bc = O.baseline_bc()
    lv = levels_for(n)
    rtol = oracle_rtol(O, K_np, bc)
    times, iters = [], None
    t_all = time.perf_counter()
    for _ in range(reps):
        t = time.perf_counter()
        h, res = O.solve_head_pcg(K_np, bc, lv, max_iter=500, check_every=1, rtol=rtol)
        O.velocity(h, K_np, bc)
        times.append(time.perf_counter() - t)
        note(f"oracle solve {len(times)}: {times[-1]:.2f} s, {res.iterations} iterations")
        iters = res.iterations
        if time.perf_counter() - t_all > budget_s * (len(times) + 1) / (reps + 1):
            break
    sec = statistics.median(times)
    return {"value": round(1.0 / sec, 4), "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"median of {len(times)} full oracle solves at {n}^3 (set-up + PCG to "
                      f"||r||/||b|| <= 1e-10, {iters} iterations, + velocity): {sec:.2f} s per solve",
            "iterations": iters}


def roofline(prof, hbm, src, precision):
    """Dominant kernel by time per PCG iteration; achieved = algorithmic bytes / launch time.
    traffic: the DRAM bytes of one launch of that kernel in this precision's solver, from an ncu
    capture summarised in profiles/traffic.json (keyed by V-cycle precision, then kernel)."""
    best = None
    for name, ms, nbytes, per_iter in prof:
        if nbytes <= 0 or per_iter <= 0:
            continue
        tot = ms * per_iter
        if best is None or tot > best[0]:
            best = (tot, name, ms, nbytes)
    if best is None:
        return None
    _, name, ms, nbytes = best
    ach = nbytes / (ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(precision, {}).get(name)
    return {"kernel": name, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(ach / hbm, 4), "peak_source": src, "traffic": traffic,
            "alg_bytes_per_launch": nbytes, "ms_per_launch": round(ms, 5)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS),
                    help="c2: 256^3 sigma2 4 lambda 8 (default); c1: 64^3 sigma2 1 lambda 4; "
                         "c3: 512^3 sigma2 1 lambda (16, 16, 4)")
    ap.add_argument("--size", type=int, default=None, help="grid edge (overrides the config's)")
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-kernels", action="store_true", help="print per-kernel timings")
    ap.add_argument("--seed", type=int, default=20240601)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched Monte Carlo ensemble")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm start records")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="run only the batched Monte Carlo ensemble and print its record")
    ap.add_argument("--ensemble-count", type=int, default=128)
    ap.add_argument("--no-graph", action="store_true",
                    help="host-driven PCG loop instead of the CUDA-graph while loop (for profilers)")
    args = ap.parse_args()
    global USE_GRAPH
    USE_GRAPH = 0 if args.no_graph else 1
    args.warmup = max(args.warmup, 3)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist_ctx = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        dist_ctx = dist
    else:
        torch.cuda.set_device(0)
    n, sigma2, lam = CONFIGS[args.config]
    if args.size is not None:
        n = args.size
    if args.config != "c2":  # the ensemble (C4) and warm-start (C5) records go with the headline run
        args.no_ensemble = args.no_learned = True
    lam_s = "x".join(f"{v:g}" for v in lam) if isinstance(lam, tuple) else f"{lam:g}"
    config = {"workload": f"darcy_ccmg_pcg_{n}^3_sigma2_{sigma2:g}_lambda_{lam_s}",
              "grid": [n, n, n], "cells": n ** 3, "lnK": "gaussian, exponential covariance, 1000 modes",
              "tolerance": "||b-Ah||/||b|| <= 1e-10", "bc": "h=1 at x=0, h=0 at x=L, no-flow elsewhere",
              "step": "set-up from K + PCG + face velocity", "l2": "inputs larger than L2 (no flush)",
              "parallelism": f"replicas{world}" if world > 1 else "single"}
    hbm, src = peaks()

    if args.impl == "reference":
        if rank != 0:
            if dist_ctx is not None:
                dist_ctx.destroy_process_group()
            return
        print(json.dumps(reference_arm(args, n, sigma2, lam, config)), flush=True)
        if dist_ctx is not None:
            dist_ctx.destroy_process_group()
        return

    import macroflow3d_b200 as M
    from macroflow3d_b200 import build
    build.build_lib()
    prec = {"fp64": M.PREC_FP64, "fp32": M.PREC_FP32, "bf16": M.PREC_BF16}[args.precision]
    if args.ensemble_only:
        if rank == 0:
            with Clocks(torch.cuda.current_device()) as clk:
                ens = ensemble_steps(M, prec, args.ensemble_count, args.steps, args.warmup, args.seed)
            ens["clocks"] = clk.summary()
            print(json.dumps({"metric": "ensemble_solves_per_s", "value": ens["batched_solves_per_s"],
                              "unit": "solves/s", "ensemble": ens}), flush=True)
        if dist_ctx is not None:
            dist_ctx.barrier()
            dist_ctx.destroy_process_group()
        return
    K = make_K(M, n, sigma2, lam, replica_seed(args.seed, rank), torch.cuda.current_device())
    torch.cuda.synchronize()

    note(f"{n}^3 {args.precision}: {args.warmup} warm-up + {args.steps} timed steps")
    with Clocks(torch.cuda.current_device()) as clk:
        out = run_steps(M, n, K, prec, args.steps, args.warmup, dist_ctx)
    clocks = clk.summary()
    ms = out["ms_total"]
    if dist_ctx is not None:
        ms = max_over_ranks(dist_ctx, ms, "cuda")
    value = replicas_value(world, args.steps, ms)
    res = out["res"]
    line = {"metric": f"darcy_solves_per_s_{n}cubed_relres_1e-10", "value": round(value, 4),
            "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer / f32 V-cycle" if prec == M.PREC_FP32 else args.precision,
            "data": "synthetic (seeded randomization-method lnK field)", "config": config}
    line["iterations"] = out["iters"][-1]
    line["true_rel_residual"] = res.true_rel_residual
    line["cell_updates_per_s"] = round(n ** 3 * out["iters"][-1] * value, 1)
    line["gpu_launches"] = out["launches"] * args.steps
    line["clocks"] = clocks

    if rank == 0:
        prof = out["solver"].profile(reps=10)
        line["roofline"] = roofline(prof, hbm, src, args.precision)
        if args.profile_kernels:
            line["kernels"] = [{"name": a, "ms": round(b, 5), "GBps": round(c / (b * 1e-3) / 1e9, 1) if b > 0 else None,
                                "per_iter": d} for a, b, c, d in prof]
    out["solver"].close()

    if not args.no_fp64_compare and prec != M.PREC_FP64:
        note("plain FP64 solver on the same field")
        o64 = run_steps(M, n, K, M.PREC_FP64, args.steps, args.warmup, dist_ctx)
        ms64 = o64["ms_total"]
        line["fp64_plain"] = {"solves_per_s": round(world * args.steps / (ms64 / 1e3), 4),
                              "iterations": o64["iters"][-1],
                              "true_rel_residual": o64["res"].true_rel_residual}
        d = (out["h"] - o64["h"]).abs().max().item() / o64["h"].abs().max().item()
        line["head_rel_maxdiff_vs_fp64"] = d
        line["speedup_vs_fp64_plain"] = round(value / line["fp64_plain"]["solves_per_s"], 3)
        iters64 = o64["iters"][-1]
        o64["solver"].close()
    else:
        iters64 = out["iters"][-1]

    if rank == 0 and world == 1 and not args.no_e2e:
        note("end to end through host buffers")
        K_host = K.cpu().pin_memory()
        # a pipelined run: the first upload and the last download are not overlapped, so the
        # run is long enough (at least 20 steps) for them not to dominate the throughput
        e2e_n = max(20, args.steps)
        v, bi, bo = e2e_steps(M, n, K_host, prec, e2e_n, 2)
        line["e2e"] = {"value": round(v, 4), "unit": "solves/s", "h2d_bytes_per_step": bi,
                       "d2h_bytes_per_step": bo, "steps": e2e_n,
                       "copies": "second stream, double-buffered: the next K up and the previous head "
                                 "down while a step solves"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        note(f"CPU baseline on {host_cores()} cores")
        line["cpu_baseline"] = cpu_baseline(K.cpu().numpy(), n)
    if rank == 0 and world == 1 and not args.no_learned:
        note("learned initial guess")
        ws = M.WarmStart.pretrained()
        ol = run_steps(M, n, K, prec, args.steps, args.warmup, None, warmstart=ws)
        v_l = args.steps / (ol["ms_total"] / 1e3)
        line["learned_mixed"] = {"solves_per_s": round(v_l, 4), "iterations": ol["iters"][-1],
                                 "true_rel_residual": ol["res"].true_rel_residual,
                                 "step": "set-up from K + network inference + PCG from its guess + face velocity",
                                 "speedup_vs_fp64_plain": round(v_l / line["fp64_plain"]["solves_per_s"], 3)
                                 if "fp64_plain" in line else None,
                                 "speedup_vs_mixed": round(v_l / value, 3)}
        ol["solver"].close()
        ws.close()
        note("learned initial guess on held-out fields")
        line["warm_start_c5"] = warmstart_eval(M, prec, args.seed)
    if rank == 0 and world == 1 and not args.no_ensemble:
        del K
        torch.cuda.empty_cache()
        note(f"ensemble of {args.ensemble_count} realisations (child process)")
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--ensemble-only", "--steps", "3", "--warmup", "3",
               "--seed", str(args.seed), "--ensemble-count", str(args.ensemble_count),
               "--precision", args.precision] + (["--no-graph"] if args.no_graph else [])
        line["ensemble"] = ensemble_isolated(cmd, ENSEMBLE_TIMEOUT_S)

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist_ctx is not None:
        dist_ctx.barrier()
        dist_ctx.destroy_process_group()


def reference_arm(args, n, sigma2, lam, config):
    """The reference's stock solve_head(PCG_MG) + compute_velocity_from_head, from oracle/_ref.
    K comes from the oracle's host generator (the same modes and evaluation as this library's),
    so this process loads only the reference build and the oracle."""
    import numpy as np
    from oracle import oracle as O
    base = {"impl": "reference", "metric": f"darcy_solves_per_s_{n}cubed_relres_1e-10", "unit": "solves/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded randomization-method lnK field)", "config": config}
    O.set_threads(host_cores())
    lams = tuple(lam) if isinstance(lam, (tuple, list)) else (lam, lam, lam)
    K = O.generate_K((n, n, n), sigma2, lams, seed=args.seed, n_modes=1000)
    bc = O.baseline_bc()
    rtol = oracle_rtol(O, K, bc)
    if O.ref_available():
        ms, it, conv, _, _, _ = O.ref_bench(K, bc, levels_for(n), 500, 1, rtol, args.warmup, args.steps)
        total = float(np.sum(ms))
        value = args.steps / (total / 1e3)
        base.update({"value": round(value, 4), "ms_per_step": round(total / args.steps, 3),
                     "iterations": it, "converged": conv,
                     "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": 0,
                                      "kind": "reference",
                                      "sample": "the reference's CUDA solve_head + velocity (built from its "
                                                "sources into oracle/_ref), full solves on one B200"},
                     "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        return base
    # the reference was not built: the oracle port on the host cores
    cb = cpu_baseline(K, n)
    base.update({"value": cb["value"], "ms_per_step": round(1e3 / cb["value"], 3), "cpu_baseline": cb,
                 "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    return base


if __name__ == "__main__":
    main()
