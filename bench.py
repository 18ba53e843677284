"""Benchmark of the ensemble membrane solid time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cvfes_b200|reference]
                    [--workload tube256x1024] [--precision fp32|fp64]
                    [--state auto|previous|velocity] [--legs main,adjoint,batched]

A step is one explicit time step of every sample of the workload.  Default
workload: the 256 x 1024-node tube (262,144 nodes, 523,776 triangles), 512 GMRF
samples, dt = 5e-7, FP32 state (velocity-state form); K = 2000 steps (the workload's
run length).

Metric: sample-timesteps/s = samples x steps / seconds, whole job.

* ``value``: CUDA events around ``GPUSolidSolver.Advance`` of the K steps with the
  state resident in HBM: replays of a captured CUDA graph of ``--chunk`` steps when
  K >= the chunk, plain launches from one library call for the rest (all of it when
  K < chunk).  The state (3 x 1.6 GB) is larger than L2, so no flush is needed.
* ``e2e``: ``--e2e-steps`` steps through the reference's per-step API, as
  ``TransientSolverGPU`` drives it: ``RefreshContext(fluid)`` (the pressure of time
  t, passed to the step kernel as a launch argument, 8 bytes) then ``Solve(t, dt)``,
  then ``Norms(out=pinned)`` -- the FP64 per-sample norms and the non-finite
  watchdog read back into pinned host memory, which synchronises every step.  The
  solver runs with ``norms_every = 1``: the persistent fan kernel accumulates the norms
  while it writes the new state, so they cost no second pass over the state
  (``--separate-norms``: the separate pass instead).
* ``adjoint`` (default line): forward + adjoint gradient evaluations of the
  64 x 128 tube, 64 samples, 500 steps (FP32 and FP64): gradients/s, the ratio
  (fwd + adj) / fwd and the reverse pass's bandwidth.
* ``batched`` (default line): the uneven 64-tube ensemble (FP32) advanced by the
  batched kernels, sample-timesteps/s summed over the tubes.

``--impl reference`` times the reference's own CPU path of the step (its compiled
``MultiplyByVector`` plus the NumPy update and Dirichlet rows of
``physicsSolver.py:263-292``, with ``OMP_NUM_THREADS`` = the host's cores) on a few
of the workload's samples; its inputs (mesh, the same GMRF sample columns, the same
mass lumping) come from the oracle's restatement, so the reference arm loads no
product library.  Multi-GPU: each rank advances its own independent ensemble
(samples do not interact), no collectives on the data path; timing is the max over
ranks.
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


def algorithmic_bytes(N, E, S, b, bt, state="previous"):
    """Bytes one step must move: per sample u_n, u_{n-1} read, u_{n+1} written (9N),
    inverse mass (N), element coefficient (E); shared: int32 connectivity (12 B per
    element), a 45-entry symmetric template per element and the unit load (3N).  The
    velocity-state form reads u_n and v_n and writes u_{n+1} and v_{n+1} (12N)."""
    per_node = 13 if state == "velocity" else 10
    return S * b * (per_node * N + E) + E * (12 + 45 * bt) + 3 * N * bt


def adjoint_bytes(N, E, S, b, bt, log_h):
    """Bytes one reverse step must move: per sample u_n, u_{n+1} read and u_{n-1}
    written (backward reconstruction, 9N), chi_{n+1}, chi_{n+2} read and chi_n written
    (9N), inverse mass (N), coefficient (E), the Gamma accumulator read and written
    (2E) and, for log h, the G accumulator (2N); shared data as in the forward step."""
    return S * b * (19 * N + 3 * E + (2 * N if log_h else 0)) + E * (12 + 45 * bt) + 3 * N * bt


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


def workload_config(args, case, world):
    """The workload description both arms print (the same dict, key for key)."""
    N, E = case.nc * case.na, 2 * case.nc * (case.na - 1)
    return {"workload": args.workload, "nodes": N, "elements": E, "samples": case.n_samples,
            "dt": case.dt, "run_steps": case.n_steps, "mass_lumping": case.mass_lumping,
            "material": "per-element GMRF E and h, seeds %d/%d" % (case.seed_E, case.seed_h),
            "parallelism": f"replicas{world}",
            "l2": "per-step state and coefficients > 126 MB L2, no flush"}


# ------------------------------------------------------------------ reference arm
def reference_inputs(case, n_cols):
    """Mesh and material of the first ``n_cols`` samples of ``case``'s ensemble, made
    without the product library: the tube geometry (plain NumPy) and the oracle's
    restatement of the GMRF sampler (the same columns the GPU arm's ensemble has)."""
    from cvfes_b200.mesh import tube_mesh
    from oracle.gmrf_oracle import material
    nodes, elems, inlet, outlet = tube_mesh(case.geometry())
    E_, h = material(elems, len(nodes), case.n_samples, np.arange(n_cols), case.seed_E,
                     case.seed_h, case.E0, case.sigma_logE, case.h0, case.sigma_logh, case.tau)
    coefK = E_ * h
    gthick = np.repeat(h[:, :, None], 3, axis=2)
    # row-sum lumping is the reference's own lumping with 3 rho (its assembly applies the
    # quadrature weight twice, physicsSolver.py:197 and optimizedSolidAssemble.pyx:564-566)
    rho = case.density * (3.0 if case.mass_lumping == "rowsum" else 1.0)
    return nodes, elems, np.concatenate([inlet, outlet]), coefK, gthick, rho


def cpu_reference_run(case, S_cpu, n_steps, warmup, threads=None):
    """Time the reference's CPU solid step (its compiled MultiplyByVector plus the NumPy
    update of physicsSolver.py:263-292) on S_cpu samples of the workload."""
    from oracle import solid_oracle as so
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    nodes, elems, bdy, coefK, gthick, rho = reference_inputs(case, S_cpu)
    ref = so.load_reference_module()
    kind = "reference" if ref is not None else "port"
    if case.dt is None:
        raise SystemExit("the reference arm needs a workload with a fixed dt")
    o = so.OracleSolidSolver(nodes, elems, bdy, coefK, gthick, rho, case.nu, case.damp, case.dt,
                             backend="reference" if ref is not None else "numpy")
    pres = case.pressures(warmup + n_steps)
    for n in range(warmup):
        o.step(pres[n])
    t0 = time.perf_counter()
    for n in range(warmup, warmup + n_steps):
        o.step(pres[n])
    dt = time.perf_counter() - t0
    return S_cpu * n_steps / dt, kind, dt


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank, world, _ = dist_setup(args)
    if rank != 0:
        return 0
    from cvfes_b200.cases import CASES
    case = CASES[args.workload]
    cores = os.cpu_count()
    S_cpu = args.cpu_samples
    value, kind, secs = cpu_reference_run(case, S_cpu, args.steps, args.warmup, cores)
    sample = (f"samples 0..{S_cpu - 1} of the {case.n_samples}-sample ensemble, {args.steps} "
              f"steps after {args.warmup} warm-up; samples never interact, so sample-timesteps/s "
              f"is linear in the sample count")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, case, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "cpu": cpu_model(), "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
class _Clock:
    """The fluid solver's time as ``RefreshContext`` reads it (``physicSolver.t``)."""
    t = 0.0


def gpu_main(args, case, rank, world, local, dev):
    import torch
    import torch.distributed as dist
    from cvfes_b200.cases import P_MAX, RAMP_STEPS, build_mesh
    from cvfes_b200.replicas import max_over_ranks, rank_case
    from cvfes_b200.solver import GPUSolidSolver, LocalComm

    prec = 32 if args.precision == "fp32" else 64
    mesh = build_mesh(rank_case(case, rank))
    S, N, E = mesh.nSmp, mesh.nNodes, mesh.nElements
    dt = case.dt

    class Cfg:
        nSmp = S
        # norms_every 1: each Solve also produces the FP64 norms of its new state in the
        # same kernel pass (the e2e leg reads them back every step)
        gpu = type("G", (), dict(precision=prec, use_graph=True, graph_chunk=args.chunk,
                                 watchdog=True, device=local, state=args.state,
                                 norms_every=0 if args.separate_norms else 1))()
        dt_f = 0.01
        exportBdyStressFilename = None
        useConstantStress = False
        # the workload's schedule p_n = P min(n / 100, 1) as RefreshContext's linear ramp
        constant_pressure = P_MAX
        pressure_ramp = "linear"
    Cfg.dt = dt
    Cfg.constant_T = RAMP_STEPS * dt

    solver = GPUSolidSolver(LocalComm(), mesh, Cfg)
    from cvfes_b200 import _lib
    variant = _lib.get_step_tuning(prec)["staged"]
    kernel = {0: "k_step", 1: "k_step_staged", 2: "k_step_gather", 3: "k_step_fan",
              4: "k_step_pipe", 5: "k_step_burst", 6: "k_step_fanp", 7: "k_step_tile",
              8: "k_step_fan (two ahead)"}.get(variant, str(variant))
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
    ck = clocks.summary(t_wall0, t_wall1)
    ms_max = max_over_ranks(ms, dev)
    chunk = args.chunk
    used_graph = K >= chunk
    launches = K + (K // chunk + (1 if K % chunk else 0) if used_graph else 1)
    nrm = solver.Norms(check_finite=False)
    finite = bool(np.all(nrm[:, 3] == 0))

    # e2e through the per-step public API: RefreshContext + Solve, norms out every step
    K2 = args.e2e_steps
    n_host = torch.empty((S, 4), dtype=torch.float64, pin_memory=True)
    fluid = _Clock()
    n0 = max(W, args.chunk) + K  # schedule position after the warm-up and timed steps
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for j in range(K2):
        fluid.t = (n0 + j) * dt
        solver.RefreshContext(fluid)
        solver.Solve(fluid.t, dt)
        solver.Norms(out=n_host)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.stop()
    ms2 = max_over_ranks(e0.elapsed_time(e1), dev)
    if world > 1:
        dist.barrier()
    solver.release_graphs()

    b = 4 if prec == 32 else 8
    bstep = algorithmic_bytes(N, E, S, b, b, solver.state_form)
    peaks, peak_kind = measured_peaks()
    achieved = bstep / (ms / K * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(f"{args.workload}_fp{prec}_{solver.state_form}")
    out = {
        "value": world * S * K / (ms_max * 1e-3), "ms_per_step": ms_max / K,
        "dtype": "f32" if prec == 32 else "f64",
        "run": {"state_form": solver.state_form, "graph_chunk": chunk,
                "graph_replays": used_graph, "finite": finite},
        "e2e": {"value": world * S * K2 / (ms2 * 1e-3), "unit": UNIT, "steps": K2,
                "path": "RefreshContext + Solve + Norms(out=pinned) per step" +
                        (" (norms by a separate pass)" if args.separate_norms else
                         " (norms fused into the step kernel)"),
                "h2d_bytes_per_step": 8, "d2h_bytes_per_step": S * 4 * 8 + 8},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "traffic": traffic, "peak_source": peak_kind, "bytes_per_step": bstep},
        "clocks": ck,
    }
    del solver
    torch.cuda.empty_cache()
    return out


def measure_adjoint(args, workload, prec, rank, world, local, dev, evals, warm):
    """Forward + adjoint gradient evaluations of the mismatch objective; one evaluation
    is T forward steps, then T reverse steps and the gradient."""
    import torch
    from cvfes_b200.adjoint import wall_mismatch
    from cvfes_b200.cases import CASES, adjoint_setup
    from cvfes_b200.replicas import max_over_ranks, rank_case

    case = CASES[workload]
    problem, logE, logh, _ = adjoint_setup(rank_case(case, rank), precision=prec, device=dev)
    S, N, E, T = problem.S, problem.N, problem.E, problem.T
    log_h = problem.grad_logh
    logE_d, logh_d = logE.to(dev), logh.to(dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warm):
        problem.objective(logE_d, logh_d)
        problem.gradient()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local).start()
    time.sleep(0.6)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(3 * evals)]
    t0 = time.perf_counter()
    for k in range(evals):
        evs[3 * k].record(stream)
        problem.objective(logE_d, logh_d)
        evs[3 * k + 1].record(stream)
        problem.gradient()
        evs[3 * k + 2].record(stream)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    clocks.stop()
    fwd = sum(evs[3 * k].elapsed_time(evs[3 * k + 1]) for k in range(evals))
    adj = sum(evs[3 * k + 1].elapsed_time(evs[3 * k + 2]) for k in range(evals))
    ms_tot, ms_fwd, ms_adj = (max_over_ranks(x, dev) for x in (fwd + adj, fwd, adj))
    finite = bool(torch.isfinite(problem.J).all())

    # e2e through the autograd.Function with host tensors in and gradients out
    lE_h = logE.to(torch.float64).pin_memory()
    lh_h = logh.to(torch.float64).pin_memory()
    gE_h = torch.empty_like(lE_h).pin_memory()
    gh_h = torch.empty_like(lh_h).pin_memory() if log_h else None
    J_h = torch.empty(S, dtype=torch.float64).pin_memory()
    K2 = max(1, min(evals, 2))
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
    del problem
    torch.cuda.empty_cache()

    b = 4 if prec == 32 else 8
    b_fwd = algorithmic_bytes(N, E, S, b, b)
    b_rev = adjoint_bytes(N, E, S, b, b, log_h)
    peaks, peak_kind = measured_peaks()
    achieved = b_rev / (ms_adj / evals / T * 1e-3) / 1e9
    return {
        "workload": workload, "dtype": "f32" if prec == 32 else "f64", "nodes": N,
        "elements": E, "samples": S, "time_steps": T, "params": "logE,logh" if log_h else "logE",
        "evaluations": evals, "warmup": warm, "finite": finite,
        "value": world * S * T * evals / (ms_tot * 1e-3), "unit": "sample-timesteps/s (fwd+adjoint)",
        "gradients_per_s": world * S * evals / (ms_tot * 1e-3),
        "fwd_ms": ms_fwd / evals, "adj_ms": ms_adj / evals,
        "ratio_fwd_plus_adj_over_fwd": ms_tot / ms_fwd,
        "e2e": {"value": world * S * T * K2 / (ms_e2e * 1e-3), "unit": UNIT,
                "path": "wall_mismatch autograd.Function, host logE/logh in, gradients out",
                "h2d_bytes_per_step": 2 * E * S * 8,
                "d2h_bytes_per_step": (2 if log_h else 1) * E * S * 8 + S * 8},
        "roofline": {"bound": "hbm", "kernel": "k_reverse (reverse pass, per step)",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peak_kind,
                     "bytes_per_step": b_rev},
        # forward: T steps, T / obs_every mismatch launches, checkpoint copies and set-up;
        # reverse: T steps, T / obs_every forcing launches and the gradient reduction
        "gpu_launches_per_evaluation": (T + T // problem_obs_every(case) + 2 * T // 48 + 4) +
                                       (T + T // problem_obs_every(case) + 1),
        "clocks": clocks.summary(t0, t1),
    }


def problem_obs_every(case):
    return int(case.extra.get("obs_every", 10))


def measure_batched(args, prec, rank, world, local, dev, steps, warm, meshes_cases=None):
    """64 uneven tubes (own resolution, radius, length, sample count and CFL time step)
    advanced by one persistent launch per launch group and step."""
    import torch
    from cvfes_b200.batched import BatchedSolidSolver
    from cvfes_b200.cases import P_MAX, RAMP_STEPS, case_dt
    from cvfes_b200.replicas import max_over_ranks
    from cvfes_b200.tune import tune_batch

    cases, meshes = meshes_cases
    dts = [case_dt(c, m) for c, m in zip(cases, meshes)]
    batch = BatchedSolidSolver(meshes, dts, precision=prec, device=dev, graph_chunk=48,
                               state=args.state)
    tuned = tune_batch(batch)
    pres = P_MAX * np.minimum(np.arange(warm + steps, dtype=np.float64) / RAMP_STEPS, 1.0)
    stream = torch.cuda.current_stream(dev)
    batch.Advance(pres[:warm])
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local).start()
    time.sleep(0.6)
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    batch.Advance(pres[warm:warm + steps])
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, dev)
    finite = all(bool(np.all(n[:, 3] == 0)) for n in batch.Norms(check_finite=False))
    S_total = batch.sample_count()
    bstep = batch.algorithmic_bytes()
    peaks, peak_kind = measured_peaks()
    achieved = bstep / (ms / steps * 1e-3) / 1e9
    n_groups = len(batch.groups)
    out = {
        "workload": "batched64", "dtype": "f32" if prec == 32 else "f64",
        "tubes": len(meshes), "nodes": sum(m.nNodes for m in meshes),
        "elements": sum(m.nElements for m in meshes), "samples": S_total,
        "steps": steps, "warmup": warm, "finite": finite, "state_form": batch.state_form,
        "value": world * S_total * steps / (ms_max * 1e-3), "unit": UNIT,
        "ms_per_step": ms_max / steps,
        "kernel": "fan" if batch.variant == 1 else "row gather", "vec": tuned.get("vec"),
        "grid": tuned.get("grid"), "launch_groups": n_groups,
        "gpu_launches": n_groups * (steps + steps // batch.graph_chunk + 1),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "peak_source": peak_kind, "bytes_per_step": bstep},
        "clocks": clocks.summary(t0, t1),
    }
    batch.release_graphs()
    del batch
    torch.cuda.empty_cache()
    return out


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from cvfes_b200.cases import CASES, batched_cases, build_meshes

    rank, world, local = dist_setup(args)
    legs = set(args.legs.split(","))
    meshes_cases = None
    if "batched" in legs:
        # the batch's GMRF material in a spawn pool, before any CUDA work of this process
        cases = batched_cases(64, seed=7 + 1000 * rank)
        meshes_cases = (cases, build_meshes(cases))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    case = CASES[args.workload]
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic",
            "config": workload_config(args, case, world)}
    if "main" in legs:
        line.update(gpu_main(args, case, rank, world, local, dev))
    if "adjoint" in legs:
        line["adjoint"] = {
            "fp32": measure_adjoint(args, "adjoint64", 32, rank, world, local, dev,
                                    args.adj_evals, 1),
            "fp64": measure_adjoint(args, "adjoint64", 64, rank, world, local, dev,
                                    args.adj_evals, 1)}
    if "batched" in legs:
        line["batched"] = measure_batched(args, 32, rank, world, local, dev, args.batch_steps,
                                          48, meshes_cases)
    if rank == 0 and world == 1 and "main" in legs and not args.no_cpu_baseline:
        v, kind, secs = cpu_reference_run(case, args.cpu_samples, args.cpu_steps, 1,
                                          os.cpu_count())
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": kind, "cpu": cpu_model(),
            "sample": f"samples 0..{args.cpu_samples - 1} of the {case.n_samples}-sample "
                      f"ensemble, {args.cpu_steps} steps after 1 warm-up, reference "
                      f"MultiplyByVector + NumPy update (linear in the sample count)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_workload(args):
    """A single non-default workload as its own line (adjoint or batched)."""
    import torch
    import torch.distributed as dist
    from cvfes_b200.cases import CASES, batched_cases, build_meshes

    rank, world, local = dist_setup(args)
    meshes_cases = None
    if args.workload == "batched64":
        cases = batched_cases(64, seed=7 + 1000 * rank)
        meshes_cases = (cases, build_meshes(cases))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=dev)
    prec = 32 if args.precision == "fp32" else 64
    if args.workload == "batched64":
        r = measure_batched(args, prec, rank, world, local, dev, args.steps, args.warmup,
                            meshes_cases)
        metric = METRIC
        cfg = {"workload": "batched64", "tubes": r["tubes"], "nodes": r["nodes"],
               "elements": r["elements"], "samples": r["samples"],
               "parallelism": f"replicas{world}"}
    else:
        r = measure_adjoint(args, args.workload, prec, rank, world, local, dev, args.steps,
                            args.warmup)
        metric = "sample-timesteps/s (fwd+adjoint)"
        c = CASES[args.workload]
        cfg = {"workload": args.workload, "nodes": r["nodes"], "elements": r["elements"],
               "samples": r["samples"], "time_steps": r["time_steps"], "params": r["params"],
               "parallelism": f"replicas{world}",
               "step": "one gradient evaluation (T forward + T reverse time steps)",
               "obs_every": problem_obs_every(c)}
    if rank == 0:
        line = {"metric": metric, "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": r["dtype"], "data": "synthetic",
                "config": cfg, "result": r, "roofline": r["roofline"], "clocks": r["clocks"]}
        if "e2e" in r:
            line["e2e"] = r["e2e"]
        print(json.dumps(line), flush=True)
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
    ap.add_argument("--state", default="auto", choices=["auto", "previous", "velocity"])
    ap.add_argument("--chunk", type=int, default=48)
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--legs", default="main,adjoint,batched",
                    help="legs of the default line: main, adjoint, batched")
    ap.add_argument("--adj-evals", type=int, default=3)
    ap.add_argument("--batch-steps", type=int, default=96)
    ap.add_argument("--cpu-samples", type=int, default=4)
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--separate-norms", action="store_true",
                    help="e2e: norms by a separate pass instead of fused into the step")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.chunk % 6:
        raise SystemExit("--chunk must be a multiple of 6")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("batched64", "adjoint64", "stenosed512x2048", "stenosed256x512"):
        return run_workload(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
