"""Autotuner for the time step's launch configuration.

Knobs (all leave the neighbour sets and cell lists bit-exact):
* the pair-pass family (`epp_set_tuning`): 0 = warp-tile search + list passes, 1 = one warp per
  occupied cell, 2..32 = lanes per particle (family changes round at the FP32 level only);
* the threads per block of the family-0 passes (`epp_set_block_threads`): 128, 64 or 32 -- small
  systems spread over more SMs with smaller blocks (no change in results).

The re-sort cadence is not a knob: the reference re-sorts every step and the cell lists are
compared bit-exactly per step, so the cadence is 1.

A configuration is tuned on a representative dam break of the same dimension and size bucket
(particle count rounded to a quarter decade), timed over a few steps, and cached in a JSON file
keyed by GPU name, dimension, size bucket and mode.  Batches (more than one instance) use family 0
and tune the block size only.  Two objectives: "single" is one run's time per step (the plain
path); "concurrent" is the time per step per run of several copies stepped together on their own
streams (serving, where many runs share the GPU): a family that wins alone by launching fewer,
wider kernels can lose once the GPU is full.
"""
import json
import math
import os
import time

from . import abi, casegen

FAMILIES = (0, 4, 8, 1)
THREADS = (128, 64, 32)
SYM = abi.EPP_CRITERION_SYMMETRY
CONT = abi.EPP_ACTION_DAMBREAK_CONTINUITY


def size_bucket(n):
    """Particle count rounded to a quarter decade (10^(k/4))."""
    return int(round(4 * math.log10(max(n, 1))))


def candidates(batch=False):
    fam = (0,) if batch else FAMILIES
    out = []
    for f in fam:
        for t in (THREADS if f == 0 else (128,)):
            out.append((f, t))
    return out


def default_cache_path():
    return os.environ.get("EPP_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "epp", "tune.json")


class TuneCache:
    """JSON cache {key: {"family": f, "threads": t, "ms": {...}}}."""

    def __init__(self, path=None):
        self.path = path or default_cache_path()
        self.data = {}
        if os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.data = json.load(f)
            except (OSError, ValueError):
                self.data = {}

    @staticmethod
    def key(gpu, dim, n, batch, concurrent=0):
        mode = "batch" if batch else "concurrent%d" % concurrent if concurrent > 1 else "single"
        return "%s|%dD|b%d|%s" % (gpu, dim, size_bucket(n), mode)

    def get(self, key):
        return self.data.get(key)

    def put(self, key, entry):
        self.data[key] = entry
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def time_config(ctx, phys, family, threads, steps=20, warmup=3):
    """Host-clock ms per step of `steps` fused steps after `warmup`, with this configuration."""
    ctx.set_tuning(family)
    if family == 0:
        ctx.set_block_threads(threads)
    ctx.step(warmup, phys)
    ctx.synchronize(raise_on_status=False)
    t0 = time.perf_counter()
    ctx.step(steps, phys)
    ctx.synchronize(raise_on_status=False)
    return 1e3 * (time.perf_counter() - t0) / steps


def concurrent_copies(n, limit=16):
    """Copies stepped together when tuning for serving: enough small runs to fill the GPU, fewer
    of the large ones (about 4M particles in all)."""
    return max(1, min(limit, int(4e6 // max(n, 1))))


def time_concurrent(case, family, threads, copies, steps=20, warmup=3, device=0):
    """Host-clock ms per step per copy: `copies` contexts holding `case`, each on its own
    stream, enqueued together and waited for together."""
    from .algorithm import DeviceParticleSystem
    from .classes import NeighbourSystem
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    runs = []
    try:
        for _ in range(copies):
            d = DeviceParticleSystem(case.ps, ns, device=device)
            runs.append(d)
            d.ctx.set_tuning(family)
            if family == 0:
                d.ctx.set_block_threads(threads)
            d.syncto()
            d.ctx.search(SYM, CONT, case.physics, 0)
            d.ctx.step(warmup, case.physics)
        for d in runs:
            d.ctx.synchronize(raise_on_status=False)
        t0 = time.perf_counter()
        for d in runs:
            d.ctx.step(steps, case.physics)
        for d in runs:
            d.ctx.synchronize(raise_on_status=False)
        return 1e3 * (time.perf_counter() - t0) / (steps * copies)
    finally:
        for d in runs:
            d.close()


def tune_case(case, n_instances=1, inst=None, steps=20, device=0, timer=time_config, batch=None, concurrent=0):
    """Time every candidate on a fresh context holding `case`; returns (best, {cand: ms}).
    `batch` restricts the candidates to those a batch can use (default: n_instances > 1);
    `concurrent` > 1 times that many copies stepped together instead (time_concurrent)."""
    from .algorithm import DeviceParticleSystem
    from .classes import NeighbourSystem
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    ms = {}
    if concurrent > 1:
        for fam, thr in candidates(False):
            ms[(fam, thr)] = time_concurrent(case, fam, thr, concurrent, steps=steps, device=device)
        return min(ms, key=ms.get), ms
    for fam, thr in candidates(n_instances > 1 if batch is None else batch):
        dps = DeviceParticleSystem(case.ps, ns, device=device, n_instances=n_instances)
        if inst is not None:
            dps.ctx.set_instance_physics(*inst)
        dps.syncto()
        dps.ctx.search(SYM, CONT, case.physics, 0)
        ms[(fam, thr)] = timer(dps.ctx, case.physics, fam, thr, steps=steps)
        dps.close()
    best = min(ms, key=ms.get)
    return best, ms


def representative_case(dim, n):
    """A dam break of about n particles (fluid and walls) in the benchmark tanks."""
    if dim == 2:
        dx = math.sqrt(1.0 * 2.0 / max(n * 0.9, 1.0))
        return casegen.dam_break_2d(dx=dx, max_neighbour_number=1)
    dx = (1.0 * 1.0 * 0.6 / max(n * 0.75, 1.0)) ** (1.0 / 3.0)
    return casegen.dam_break_3d(dx=dx, max_neighbour_number=1)


class Autotuner:
    """best(dim, n, batch) -> (family, threads), from the cache or tuned once and stored."""

    def __init__(self, cache=None, device=0, gpu=None, steps=20):
        self.cache = cache if cache is not None else TuneCache()
        self.device = device
        self.steps = steps
        self._gpu = gpu

    @property
    def gpu(self):
        if self._gpu is None:
            try:
                import torch
                self._gpu = torch.cuda.get_device_name(self.device).replace(" ", "_")
            except Exception:
                self._gpu = "gpu%d" % self.device
        return self._gpu

    def best(self, dim, n, batch=False, case=None, concurrent=0):
        key = TuneCache.key(self.gpu, dim, n, batch, concurrent)
        hit = self.cache.get(key)
        if hit:
            return hit["family"], hit["threads"]
        case = case or representative_case(dim, n)
        (fam, thr), ms = tune_case(case, steps=self.steps, device=self.device, batch=batch,
                                   concurrent=0 if batch else concurrent)
        self.cache.put(key, {"family": fam, "threads": thr, "particles": case.n, "copies": max(concurrent, 1),
                             "ms_per_step": {"%d/%d" % k: v for k, v in ms.items()}})
        return fam, thr

    def cached(self, dim, n, batch=False, concurrent=0):
        """The cached choice, or None (never tunes)."""
        hit = self.cache.get(TuneCache.key(self.gpu, dim, n, batch, concurrent))
        return (hit["family"], hit["threads"]) if hit else None

    def apply(self, ctx, dim, n, batch=False, concurrent=0):
        fam, thr = self.best(dim, n, batch, concurrent=concurrent)
        ctx.set_tuning(fam)
        ctx.set_block_threads(thr)
        return fam, thr
