"""Autotuner for the step kernels: measure candidate tile shapes, keep the fastest.

Single mesh: the kernel variant, samples per thread (VEC), nodes per block and
the register bound (``cvfes_set_step_tuning``), then the fan kernel's L2 prefetch
distance (``cvfes_set_step_prefetch``).  Batch: samples per thread (the
tile's sample width, 32*VEC per warp) and the persistent grid size.  Every
candidate runs a few CUDA-graph chunks from the same saved state, timed with CUDA
events; the state is restored afterwards, so tuning does not advance the
simulation.  Results are cached in a JSON file keyed by the GPU name and the
problem's shape, so later runs of the same shape skip the measurement.
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib

STEP_CANDIDATES = {
    32: [(6, 4, 2, 2), (6, 4, 4, 2), (3, 4, 2, 2), (3, 4, 4, 2), (8, 4, 2, 2), (3, 4, 2, 1),
         (1, 4, 4, 2), (3, 2, 2, 3), (5, 4, 2, 1), (0, 4, 8, 1)],
    64: [(6, 2, 4, 2), (3, 2, 2, 2), (3, 2, 4, 2), (6, 2, 2, 2), (8, 2, 2, 2), (1, 2, 4, 2),
         (3, 1, 4, 3), (5, 1, 2, 2), (0, 2, 8, 1)],
}


def _cache_path() -> str:
    d = os.environ.get("CVFES_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cvfes_b200"))
    os.makedirs(d, exist_ok=True)
    return os.path.join(d, "tuning.json")


def _load_cache() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, value) -> None:
    c = _load_cache()
    c[key] = value
    tmp = _cache_path() + ".tmp"
    with open(tmp, "w") as f:
        json.dump(c, f, indent=1)
    os.replace(tmp, _cache_path())


def _key(kind: str, device, shape) -> str:
    name = torch.cuda.get_device_name(device)
    h = hashlib.sha1(repr(shape).encode()).hexdigest()[:16]
    return f"{kind}|{name}|{h}"


def _time_ms(fn, device) -> float:
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize(device)
    return e0.elapsed_time(e1)


def tune_step(solver, candidates: Optional[Iterable[Tuple[int, int, int, int]]] = None,
              steps: int = 96, use_cache: bool = True) -> dict:
    """Pick (variant, vec, npb, minb) for ``solver``'s precision and problem shape."""
    prec = solver.precision
    dev = solver.device
    shape = ("step", prec, solver.lclNNodes, solver.nElms, solver.nSmp, solver.plan.max_degree,
             solver.state_form)
    key = _key("step", dev, shape)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        best = cache[key]
        _lib.set_step_tuning(prec, best["vec"], best["npb"], best["staged"], best["minb"])
        _lib.set_step_prefetch(prec, **best.get("prefetch", {}))
        return dict(best, cached=True)
    saved = [b.clone() for b in solver.bufs]
    roles = (solver.cur, solver.prev, solver.nxt)
    pres = np.zeros(steps + solver.graph_chunk)

    def measure():
        solver.release_graphs()
        for b, s in zip(solver.bufs, saved):
            b.copy_(s)
        solver.cur, solver.prev, solver.nxt = roles
        solver.Advance(pres[:solver.graph_chunk])  # capture + warm
        return _time_ms(lambda: solver.Advance(pres[:steps]), dev) / steps

    # tile shapes with the automatic L2 prefetch, then the prefetch for the fastest
    # shape (fan kernel only): off, node rows only, both parts, twice as far ahead
    auto = dict(distance=-1, parts=-1)
    _lib.set_step_prefetch(prec, **auto)
    results = []
    for staged, vec, npb, minb in (candidates or STEP_CANDIDATES[prec]):
        try:
            _lib.set_step_tuning(prec, vec, npb, staged, minb)
        except _lib.CvfesError:
            continue
        ms = measure()
        results.append((ms, dict(staged=staged, vec=vec, npb=npb, minb=minb, prefetch=auto,
                                 ms_per_step=ms)))
    best = min(results, key=lambda r: r[0])[1]
    _lib.set_step_tuning(prec, best["vec"], best["npb"], best["staged"], best["minb"])
    if best["staged"] in (3, 6, 8):
        bw = solver.plan.bandwidth
        for pf in (dict(distance=0, parts=0), dict(distance=-1, parts=1),
                   dict(distance=-1, parts=3), dict(distance=2 * bw + 128, parts=3)):
            _lib.set_step_prefetch(prec, **pf)
            ms = measure()
            results.append((ms, dict(best, prefetch=pf, ms_per_step=ms)))
        best = min(results, key=lambda r: r[0])[1]
    _lib.set_step_tuning(prec, best["vec"], best["npb"], best["staged"], best["minb"])
    _lib.set_step_prefetch(prec, **best["prefetch"])
    for b, s in zip(solver.bufs, saved):
        b.copy_(s)
    solver.cur, solver.prev, solver.nxt = roles
    solver.release_graphs()
    if use_cache:
        _store(key, best)
    return dict(best, cached=False, tried=[r[1] for r in results])


def tune_batch(batch, vecs: Optional[Sequence[int]] = None,
               grids: Optional[Sequence[int]] = None, steps: int = 48,
               use_cache: bool = True, variants: Optional[Sequence[int]] = None) -> dict:
    """Pick the batch's kernel, samples per thread and persistent grid size."""
    dev = batch.device
    shape = ("batch", batch.precision, batch.state_form,
             tuple((s.lclNNodes, s.nElms, s.nSmp) for s in batch.solvers))
    key = _key("batch", dev, shape)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        best = cache[key]
        batch.set_launch(vec=best["vec"], grid=best["grid"], variant=best.get("variant", 0))
        return dict(best, cached=True)
    if variants is None:
        variants = [1, 0] if batch.totals[2] > 0 else [0]
    maxv = 4 if batch.precision == 32 else 2
    if vecs is None:
        vecs = [v for v in (4, 2, 1) if v <= maxv and all(s.nSmp % v == 0 for s in batch.solvers)]
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    grid_sets = {0: list(grids) if grids is not None else [0, 4 * sms, 8 * sms, 16 * sms],
                 1: list(grids) if grids is not None else [0, 4 * sms]}
    saved = [[b.clone() for b in s.bufs] for s in batch.solvers]
    rot0 = batch.rot
    pres = np.zeros(steps + batch.graph_chunk + 6)
    results = []
    for variant, vec, grid in [(v, x, g) for v in variants for x in vecs for g in grid_sets[v]]:
        batch.set_launch(vec=vec, grid=grid, variant=variant)
        for s, sv in zip(batch.solvers, saved):
            for b, x in zip(s.bufs, sv):
                b.copy_(x)
        batch.rot = rot0
        batch.Advance(pres[:batch.graph_chunk + 6])
        ms = _time_ms(lambda: batch.Advance(pres[:steps]), dev) / steps
        results.append((ms, dict(variant=variant, vec=vec, grid=grid, ms_per_step=ms)))
    for s, sv in zip(batch.solvers, saved):
        for b, x in zip(s.bufs, sv):
            b.copy_(x)
    batch.rot = rot0
    best = min(results, key=lambda r: r[0])[1]
    batch.set_launch(vec=best["vec"], grid=best["grid"], variant=best["variant"])
    steps0 = batch.steps
    batch.sync_roles()
    for s in batch.solvers:
        s.step_count = steps0
    if use_cache:
        _store(key, best)
    return dict(best, cached=False, tried=[r[1] for r in results])
