"""Benchmark of the ensemble membrane solid time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cvfes_b200|reference]
                    [--workload tube256x1024] [--precision fp32|fp64]

A step is one explicit time step of every sample of the workload.  Default
workload: the 256 x 1024-node tube (262,144 nodes, 523,776 triangles), 512 GMRF
samples, dt = 5e-7, FP32 state; K = 2000 steps (the workload's run length).

Metric: sample-timesteps/s = samples x steps / seconds, whole job.  ``value`` is
measured with CUDA events around the K steps (CUDA-graph replays of the fused
step kernel) with the state resident in HBM; the state (3 x 1.6 GB) is larger
than L2, so no flush is needed.  ``e2e`` runs K steps through the public
per-step API (GPUSolidSolver.Solve with the pressure copied from pinned host
memory, plus the FP64 watchdog norms read back to pinned host memory every
step).  Multi-GPU: each rank advances its own independent ensemble (samples do
not interact), no collectives on the data path; timing is the max over ranks.
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

METRIC = "sample-timesteps/s (FP32 fwd)"
UNIT = "sample-timesteps/s"


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def algorithmic_bytes(N, E, S, b, bt):
    """Bytes one step must move: per sample u_n, u_{n-1} read, u_{n+1} written (9N),
    inverse mass (N), element coefficient (E); shared: int32 connectivity (12 B per
    element), a 45-entry symmetric template per element and the unit load (3N)."""
    return S * b * (10 * N + E) + E * (12 + 45 * bt) + 3 * N * bt


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.perf_counter(), ln.strip()))

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = [ln for (t, ln) in self.lines if t0 - 0.25 <= t <= t1 + 0.25] or \
               [ln for (_, ln) in self.lines]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in rows:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus and world > 1:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    return rank, world, local


def cpu_reference_run(case, S_cpu, n_steps, warmup, threads=None):
    """Time the reference's CPU solid step (its compiled MultiplyByVector plus the NumPy
    update of physicsSolver.py:263-292) on S_cpu samples of the workload's mesh."""
    from cvfes_b200.cases import build_mesh
    from oracle import solid_oracle as so
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    mesh = build_mesh(case, n_samples=S_cpu)
    coefK, gthick = mesh.element_coefficients()
    ref = so.load_reference_module()
    kind = "reference" if ref is not None else "port"
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density, mesh.v, mesh.damp, case.dt or 5e-7,
                             backend="reference" if ref is not None else "numpy")
    pres = case.pressures(warmup + n_steps)
    for n in range(warmup):
        o.step(pres[n])
    t0 = time.perf_counter()
    for n in range(warmup, warmup + n_steps):
        o.step(pres[n])
    dt = time.perf_counter() - t0
    return S_cpu * n_steps / dt, kind, dt


def run_reference(args):
    rank, world, _ = dist_setup(args)
    if rank != 0:
        return 0
    from cvfes_b200.cases import CASES
    case = CASES[args.workload]
    cores = os.cpu_count()
    S_cpu = args.cpu_samples
    value, kind, secs = cpu_reference_run(case, S_cpu, args.steps, args.warmup, cores)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "nodes": case.nc * case.na, "samples": S_cpu,
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{S_cpu} of {case.n_samples} samples of {args.workload}, "
                                   f"{args.steps} steps after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from cvfes_b200 import _lib
    from cvfes_b200._lib import call, ptr
    from cvfes_b200.cases import CASES, build_mesh
    from cvfes_b200.solver import GPUSolidSolver, LocalComm

    rank, world, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)
    case = CASES[args.workload]
    prec = 32 if args.precision == "fp32" else 64
    from cvfes_b200.replicas import max_over_ranks, rank_case
    mesh = build_mesh(rank_case(case, rank))
    S, N, E = mesh.nSmp, mesh.nNodes, mesh.nElements

    class Cfg:
        dt = case.dt or 5e-7
        nSmp = S
        gpu = type("G", (), dict(precision=prec, use_graph=True, graph_chunk=args.chunk,
                                 watchdog=True, device=local))()
        dt_f = 0.01
        exportBdyStressFilename = None
        useConstantStress = False
        constant_T = 1.0
        constant_pressure = 0.0
        pressure_ramp = "linear"

    solver = GPUSolidSolver(LocalComm(), mesh, Cfg)
    K, W = args.steps, args.warmup
    pres = torch.from_numpy(case.pressures(W + K)).to(dev)
    stream = torch.cuda.current_stream(dev)

    # warm-up (also captures the graph)
    solver.Advance(pres[:W] if W >= args.chunk else pres[:max(W, args.chunk)])
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local).start()
    time.sleep(0.6)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t_wall0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    solver.Advance(pres[W:W + K])
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    t_wall1 = time.perf_counter()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    clocks.stop()
    ck = clocks.summary(t_wall0, t_wall1)
    ms_max = max_over_ranks(ms, dev)
    chunk = args.chunk
    launches = K + K // chunk + (1 if K % chunk else 0)

    # finite check of the result
    nrm = solver.Norms(check_finite=False)
    finite = bool(np.all(nrm[:, 3] == 0))

    # e2e through the per-step public API: host pressure in, FP64 norms out, every step
    K2 = args.e2e_steps
    p_host = torch.empty(1, dtype=torch.float64, pin_memory=True)
    p_dev = torch.empty(1, dtype=torch.float64, device=dev)
    n_host = torch.empty((S, 4), dtype=torch.float64, pin_memory=True)
    n_dev = torch.empty((S, 4), dtype=torch.float64, device=dev)
    fn_step = "cvfes_solid_step_f64" if prec == 64 else "cvfes_solid_step_f32"
    fn_norm = "cvfes_solid_norms_f64" if prec == 64 else "cvfes_solid_norms_f32"
    pv = case.pressures(W + K + K2)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s = stream.cuda_stream
    for j in range(K2):
        p_host[0] = pv[W + K + j]
        p_dev.copy_(p_host, non_blocking=True)
        call(fn_step, _lib.C.byref(solver._desc), ptr(solver.plan.coef(prec)),
             ptr(solver.plan.invm(prec)), ptr(solver.bufs[solver.cur]),
             ptr(solver.bufs[solver.prev]), ptr(solver.bufs[solver.nxt]), ptr(p_dev), None, 0,
             0.0, None, float(Cfg.dt), float(mesh.damp), s)
        solver.prev, solver.cur, solver.nxt = solver.cur, solver.nxt, solver.prev
        call(fn_norm, N, S, ptr(solver.bufs[solver.cur]), ptr(solver.bufs[solver.prev]),
             ptr(solver.plan.invm(prec)), ptr(solver.norm_work), ptr(n_dev), 0, s)
        n_host.copy_(n_dev, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms2 = max_over_ranks(e0.elapsed_time(e1), dev)
    if world > 1:
        dist.barrier()
    solver.release_graphs()

    b = 4 if prec == 32 else 8
    bstep = algorithmic_bytes(N, E, S, b, b)
    peaks, peak_kind = measured_peaks()
    achieved = bstep / (ms / K * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(f"{args.workload}_fp{prec}")

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, kind, secs = cpu_reference_run(case, args.cpu_samples, args.cpu_steps, 1,
                                              os.cpu_count())
            cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
                   "sample": f"{args.cpu_samples} of {S} samples of {args.workload}, "
                             f"{args.cpu_steps} steps, reference MultiplyByVector + NumPy update"}
        line = {
            "metric": METRIC, "value": world * S * K / (ms_max * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_max / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 32 else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "nodes": N, "elements": E, "samples": S,
                       "dt": Cfg.dt, "parallelism": f"replicas{world}",
                       "l2": "state 3x%.2f GB > L2, no flush" % (3 * N * S * b / 1e9),
                       "graph_chunk": chunk, "finite": finite},
            "e2e": {"value": world * S * K2 / (ms2 * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": 8, "d2h_bytes_per_step": S * 4 * 8},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "traffic": traffic, "peak_source": peak_kind,
                         "bytes_per_step": bstep},
            "clocks": ck,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def adjoint_bytes(N, E, S, b, bt, log_h):
    """Bytes one reverse step must move: per sample u_n, u_{n+1} read and u_{n-1}
    written (backward reconstruction, 9N), chi_{n+1}, chi_{n+2} read and chi_n written
    (9N), inverse mass (N), coefficient (E), the Gamma accumulator read and written
    (2E) and, for log h, the G accumulator (2N); shared data as in the forward step."""
    return S * b * (19 * N + 3 * E + (2 * N if log_h else 0)) + E * (12 + 45 * bt) + 3 * N * bt


def run_adjoint(args):
    """Forward + adjoint gradient evaluations of the mismatch objective; a bench step is
    one evaluation (T forward steps, then T reverse steps and the gradient)."""
    import torch
    from cvfes_b200.adjoint import wall_mismatch
    from cvfes_b200.cases import CASES, adjoint_setup

    rank, world, local = dist_setup(args)
    case = CASES[args.workload]
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=dev)
    prec = 32 if args.precision == "fp32" else 64
    from cvfes_b200.replicas import max_over_ranks, rank_case
    problem, logE, logh, _ = adjoint_setup(rank_case(case, rank), precision=prec, device=dev)
    S, N, E, T = problem.S, problem.N, problem.E, problem.T
    log_h = problem.grad_logh
    logE_d, logh_d = logE.to(dev), logh.to(dev)
    stream = torch.cuda.current_stream(dev)
    K, W = args.steps, args.warmup
    for _ in range(W):
        problem.objective(logE_d, logh_d)
        problem.gradient()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local).start()
    time.sleep(0.6)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(3 * K)]
    t0 = time.perf_counter()
    for k in range(K):
        evs[3 * k].record(stream)
        problem.objective(logE_d, logh_d)
        evs[3 * k + 1].record(stream)
        problem.gradient()
        evs[3 * k + 2].record(stream)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    clocks.stop()
    fwd = sum(evs[3 * k].elapsed_time(evs[3 * k + 1]) for k in range(K))
    adj = sum(evs[3 * k + 1].elapsed_time(evs[3 * k + 2]) for k in range(K))
    ms_tot, ms_fwd, ms_adj = (max_over_ranks(x, dev) for x in (fwd + adj, fwd, adj))
    finite = bool(torch.isfinite(problem.J).all())

    # e2e through the autograd.Function with host tensors in and gradients out
    lE_h = logE.to(torch.float64).pin_memory()
    lh_h = logh.to(torch.float64).pin_memory()
    gE_h = torch.empty_like(lE_h).pin_memory()
    gh_h = torch.empty_like(lh_h).pin_memory() if log_h else None
    J_h = torch.empty(S, dtype=torch.float64).pin_memory()
    K2 = max(1, min(K, 2))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(K2):
        lE = lE_h.to(dev, non_blocking=True).requires_grad_(True)
        lh = lh_h.to(dev, non_blocking=True).requires_grad_(log_h)
        J = wall_mismatch(lE, lh, problem)
        J.sum().backward()
        J_h.copy_(J.detach(), non_blocking=True)
        gE_h.copy_(lE.grad, non_blocking=True)
        if log_h:
            gh_h.copy_(lh.grad, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = e0.elapsed_time(e1)
    problem.release_graphs()

    b = 4 if prec == 32 else 8
    b_fwd = algorithmic_bytes(N, E, S, b, b)
    b_rev = adjoint_bytes(N, E, S, b, b, log_h)
    peaks, peak_kind = measured_peaks()
    achieved = b_rev / (ms_adj / K / T * 1e-3) / 1e9
    nck = (T + problem.ckpt_every - 1) // problem.ckpt_every
    launches_fwd = T + (T // problem.obs_every) + 2 * T // 48 + 4
    launches_rev = T + (T // problem.obs_every) + 1
    if rank == 0:
        line = {
            "metric": "sample-timesteps/s (fwd+adjoint)",
            "value": world * S * T * K / (ms_tot * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_tot / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 32 else "f64", "data": "synthetic",
            "config": {"workload": args.workload, "nodes": N, "elements": E, "samples": S,
                       "time_steps": T, "dt": problem.dt, "obs_nodes": problem.n_obs,
                       "obs_every": problem.obs_every, "ckpt_every": problem.ckpt_every,
                       "checkpoints": nck, "params": "logE,logh" if log_h else "logE",
                       "parallelism": f"replicas{world}", "l2": "state > L2, no flush",
                       "finite": finite, "step": "one gradient evaluation (T forward + T "
                                                 "reverse time steps)"},
            "adjoint": {"fwd_ms": ms_fwd / K, "adj_ms": ms_adj / K,
                        "ratio_fwd_plus_adj_over_fwd": ms_tot / ms_fwd,
                        "gradients_per_s": world * S * K / (ms_tot * 1e-3),
                        "fwd_sample_timesteps_per_s": world * S * T * K / (ms_fwd * 1e-3),
                        "fwd_bytes_per_step": b_fwd, "rev_bytes_per_step": b_rev,
                        "fwd_hbm_frac": b_fwd / (ms_fwd / K / T * 1e-3) / 1e9 / peaks["hbm_gbs"]},
            "e2e": {"value": world * S * T * K2 / (ms_e2e * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": 2 * E * S * 8,
                    "d2h_bytes_per_step": (2 if log_h else 1) * E * S * 8 + S * 8},
            "gpu_launches": K * (launches_fwd + launches_rev),
            "roofline": {"bound": "hbm", "kernel": "k_reverse (reverse pass average per step)",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                         "peak_source": peak_kind, "bytes_per_step": b_rev},
            "clocks": clocks.summary(t0, t1),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """64 uneven tubes (own resolution, radius, length, sample count and CFL time step)
    advanced by one persistent launch per step; metric summed over all tubes."""
    import torch
    import torch.distributed as dist
    from cvfes_b200.batched import BatchedSolidSolver
    from cvfes_b200.cases import P_MAX, RAMP_STEPS, batched_cases, build_meshes, case_dt
    from cvfes_b200.tune import tune_batch

    rank, world, local = dist_setup(args)
    cases = batched_cases(64, seed=7 + 1000 * rank)
    meshes = build_meshes(cases)  # spawn pool, before any CUDA work of this process
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    prec = 32 if args.precision == "fp32" else 64
    dts = [case_dt(c, m) for c, m in zip(cases, meshes)]
    batch = BatchedSolidSolver(meshes, dts, precision=prec, device=dev, graph_chunk=args.chunk)
    tuned = tune_batch(batch)
    K, W = args.steps, args.warmup
    pres = P_MAX * np.minimum(np.arange(W + K, dtype=np.float64) / RAMP_STEPS, 1.0)
    stream = torch.cuda.current_stream(dev)
    batch.Advance(pres[:W])
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local).start()
    time.sleep(0.6)
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    batch.Advance(pres[W:W + K])
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    clocks.stop()
    ms = ev0.elapsed_time(ev1)
    from cvfes_b200.replicas import max_over_ranks
    ms_max = max_over_ranks(ms, dev)
    finite = all(bool(np.all(n[:, 3] == 0)) for n in batch.Norms(check_finite=False))
    S_total = batch.sample_count()
    bstep = batch.algorithmic_bytes()
    peaks, peak_kind = measured_peaks()
    achieved = bstep / (ms / K * 1e-3) / 1e9
    # per launch group: one step kernel per step, one clock kernel per graph chunk and
    # per plain remainder
    n_groups = len(batch.groups)
    launches = n_groups * (K + K // batch.graph_chunk + 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": world * S_total * K / (ms_max * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_max / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 32 else "f64", "data": "synthetic",
            "config": {"workload": "batched64", "tubes": len(cases),
                       "nodes": sum(m.nNodes for m in meshes),
                       "elements": sum(m.nElements for m in meshes), "samples": S_total,
                       "parallelism": f"replicas{world}", "kernel": ("fan" if batch.variant == 1
                                                                    else "row gather"),
                       "vec": tuned.get("vec"), "grid": tuned.get("grid"),
                       "launch_groups": n_groups,
                       "l2": "state > L2, no flush",
                       "finite": finite},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                         "peak_source": peak_kind, "bytes_per_step": bstep},
            "clocks": clocks.summary(t0, t1),
        }
        print(json.dumps(line), flush=True)
    batch.release_graphs()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=48)
    ap.add_argument("--impl", default="cvfes_b200", choices=["cvfes_b200", "reference"])
    ap.add_argument("--workload", default="tube256x1024")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--chunk", type=int, default=48)
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--cpu-samples", type=int, default=4)
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.chunk % 3:
        raise SystemExit("--chunk must be a multiple of 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched64":
        return run_batched(args)
    if args.workload in ("adjoint64", "stenosed512x2048"):
        return run_adjoint(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
