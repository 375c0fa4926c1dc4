"""Serving loop: dam-break simulations admitted by HBM budget, resident on the device, stepped
concurrently, with completion latency per request.

The reference runs one simulation per Julia process; this is the continuous-batching form of the
same step.  Every admitted request owns a context (its state stays in HBM until it completes) and
the context's CUDA stream, so the steps of different-sized runs overlap on the device: while a
small run is bound by launch latency, a large one fills the SMs.  The host loop

* moves requests whose arrival time has passed into a FIFO queue;
* admits from the head of the queue while the resident bytes (epp_context_bytes of every live
  context) stay within the budget, so a request that arrives while others run starts as soon as
  a slot and memory free up;
* keeps a few chunks of steps queued on every resident stream, refilling a stream when
  epp_query reports it drained (non-blocking); each stream carries a CUDA priority by run size,
  so the hardware schedules the kernels of short runs first and long runs fill the rest;
* retires a run after its last step: FP64 integrals, optional download, context destroyed (the
  stream-ordered allocator returns its memory without synchronising the device).

Each request runs on its own context with the plain path's kernels and graphs, so its result is
the same whether it runs alone or in the mix.

The device calls go through a backend object, so the admission and accounting logic also runs
against a simulated backend on the CPU (tests).
"""
import collections
import math
import time

import numpy as np

from . import abi, casegen

SYM = abi.EPP_CRITERION_SYMMETRY
CONT = abi.EPP_ACTION_DAMBREAK_CONTINUITY


class RequestSpec:
    """One simulation request: dimension, fluid particle count, column aspect, steps."""

    def __init__(self, rid, arrival, dim, n_fluid, aspect, steps, column=None, dx=None):
        self.rid = rid
        self.arrival = arrival    # seconds after the start of the stream
        self.dim = dim
        self.n_fluid = n_fluid
        self.aspect = aspect
        self.steps = steps
        self.column = column      # explicit 2D column (width, height) and lattice spacing, or None
        self.dx = dx

    def expected_particles(self):
        """Fluid particles this request asks for (before the case is built)."""
        if self.column is not None:
            return int(round(self.column[0] * self.column[1] / (self.dx * self.dx)))
        return self.n_fluid

    def weight(self):
        """Expected device work: particles x steps, 3D about 2.5x 2D per particle-step."""
        return self.expected_particles() * self.steps * (2.5 if self.dim == 3 else 1.0)

    def case(self):
        """The dam break this request asks for.  2D: column 1.0 m wide, height aspect x width
        (at most 2.5 m) in the 4.0 x 3.0 m tank, dx = sqrt(W H / N).  3D: block 1.0 x 1.0 m, height
        0.4 aspect (0.2 - 1.0 m) in the 3.2 x 1.0 x 1.0 m tank, dx = cbrt(W L H / N).  A request
        with an explicit column and dx is that 2D dam break."""
        if self.column is not None:
            return casegen.dam_break_2d(dx=self.dx, column=self.column, max_neighbour_number=1)
        if self.dim == 2:
            w, h = 1.0, min(self.aspect * 1.0, 2.5)
            dx = math.sqrt(w * h / self.n_fluid)
            return casegen.dam_break_2d(dx=dx, column=(w, h), max_neighbour_number=1)
        h = 0.4 * self.aspect
        dx = (1.0 * 1.0 * h / self.n_fluid) ** (1.0 / 3.0)
        return casegen.dam_break_3d(dx=dx, column=(1.0, 1.0, h), max_neighbour_number=1)


def request_stream(n, seed=0, rate=50.0, frac_2d=0.7, n_range=(1e3, 1e6), aspect=(0.5, 2.5), steps=2000):
    """Seeded request stream: Poisson arrivals (mean `rate` per second), `frac_2d` of them 2D,
    fluid counts log-uniform in `n_range`, column aspect uniform in `aspect`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        dim = 2 if rng.random() < frac_2d else 3
        nf = int(round(math.exp(rng.uniform(lo, hi))))
        a = float(rng.uniform(aspect[0], aspect[1]))
        out.append(RequestSpec(i, t, dim, nf, a, steps))
    return out


def batch_mix_requests(n_instances=256, seed=0, dx=0.01, steps=2000, arrival=0.0):
    """The batched form's instance mix as requests (2D columns width U[0.5, 1.5] m, height
    U[1.0, 2.5] m, seed 0, dx = 0.01 m), all arriving at `arrival`."""
    cols = casegen.batch_columns(n_instances, seed)
    return [RequestSpec(k, arrival, 2, 0, None, steps, column=c, dx=dx) for k, c in enumerate(cols)]


def priority_for(n_particles):
    """Stream priority by size (lower = scheduled first): about one level per half decade, the
    smallest runs first, so short runs are not stuck behind long ones."""
    return -int(max(0, min(5, round(2 * (6.0 - math.log10(max(n_particles, 1)))))))


class Run:
    """Server-side record of one request."""

    def __init__(self, spec, case, nbytes):
        self.spec = spec
        self.case = case
        self.bytes = nbytes
        self.handle = None
        self.queued = 0          # steps enqueued on the device
        self.admitted = None     # seconds after start
        self.done = None
        self.result = None
        self.error = None

    @property
    def latency(self):
        return None if self.done is None else self.done - self.spec.arrival


class DeviceBackend:
    """Runs each request on its own epp context (own stream) on one GPU."""

    def __init__(self, device=0, download=False, priorities=True, tuner=None, tune_concurrent=True):
        self.device = device
        self.download = download
        self.priorities = priorities
        self.tuner = tuner        # autotune.Autotuner: launch configuration per dimension and size
        self.tune_concurrent = tune_concurrent   # tune for throughput with several runs resident

    def _config(self, case):
        from .classes import NeighbourSystem
        ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        adj = ns.active_pair.adjacency_matrix.tolist()
        return ns, abi.make_config(case.domain.to_abi(), case.ps.n_capacity, adj, max_neighbour_number=1,
                                   device=self.device)

    def copies(self, n):
        """Copies the tuner steps together for a run of n particles (0: tune one run alone)."""
        from .autotune import concurrent_copies
        return concurrent_copies(n) if self.tune_concurrent else 0

    def bytes_needed(self, case):
        from .lib import context_bytes
        return context_bytes(self._config(case)[1])

    def admit(self, case):
        from .algorithm import DeviceParticleSystem
        ns, _ = self._config(case)
        dps = DeviceParticleSystem(case.ps, ns, device=self.device)
        dps.physics = case.physics
        if self.priorities:
            dps.ctx.set_priority(priority_for(case.n))
        if self.tuner is not None:
            self.tuner.apply(dps.ctx, case.meta["dim"], case.n, concurrent=self.copies(case.n))
        dps.syncto()
        dps.ctx.search(SYM, CONT, case.physics, 0)
        return dps

    def enqueue(self, dps, n_steps):
        dps.ctx.step(n_steps, dps.physics)

    def idle(self, dps):
        return dps.ctx.done()

    def finish(self, dps):
        st = dps.ctx.synchronize(raise_on_status=False)
        res = {"integrals": dps.ctx.integrals(dps.physics), "status": st}
        if self.download:
            dps.asyncto()
            h = dps.host
            res["state"] = {k: h[k] for k in ("PositionVec", "VelocityVec", "Density", "Pressure", "nCount")}
        dps.close()
        return res


class Server:
    """Admission by HBM budget, resident state, continuous batching over per-request streams.

    budget_bytes: device bytes the resident contexts may hold together.
    max_active:   resident runs at most (1 = the plain path, one request at a time).
    chunk, ahead: steps per enqueue and chunks kept queued on a stream."""

    def __init__(self, backend, budget_bytes=120 * 10**9, max_active=256, chunk=100, ahead=2,
                 clock=time.perf_counter, idle_wait=50e-6):
        self.backend = backend
        self.budget = int(budget_bytes)
        self.max_active = max_active
        self.chunk = chunk
        self.ahead = ahead
        self.clock = clock
        self.idle_wait = idle_wait

    def run(self, runs):
        """Serve `runs` (Run objects with their arrival times) to completion; returns stats."""
        t0 = self.clock()
        now = lambda: self.clock() - t0  # noqa: E731
        arrivals = collections.deque(sorted(runs, key=lambda r: r.spec.arrival))
        waiting = collections.deque()
        active = []
        used = peak = 0
        max_conc = 0
        while arrivals or waiting or active:
            t = now()
            while arrivals and arrivals[0].spec.arrival <= t:
                waiting.append(arrivals.popleft())
            # FIFO admission while the head fits the budget and a slot is free
            while waiting and len(active) < self.max_active:
                r = waiting[0]
                if r.bytes > self.budget:          # can never fit: reject, keep serving the rest
                    waiting.popleft()
                    r.error = "needs %d bytes, budget %d" % (r.bytes, self.budget)
                    r.done = now()
                    continue
                if used + r.bytes > self.budget:
                    break
                waiting.popleft()
                r.handle = self.backend.admit(r.case)
                r.admitted = now()
                used += r.bytes
                peak = max(peak, used)
                active.append(r)
                self._fill(r)
            max_conc = max(max_conc, len(active))
            progressed = False
            for r in list(active):
                if not self.backend.idle(r.handle):
                    continue
                progressed = True
                if r.queued < r.spec.steps:
                    self._fill(r)
                    continue
                r.result = self.backend.finish(r.handle)
                r.handle = None
                r.done = now()
                used -= r.bytes
                active.remove(r)
            if not progressed:
                if not active and not waiting and arrivals:
                    self._sleep_until(arrivals[0].spec.arrival, now)
                else:
                    time.sleep(self.idle_wait)
        makespan = now()
        return self.stats(runs, makespan, peak, max_conc)

    def _fill(self, r):
        n = min(self.chunk * self.ahead, r.spec.steps - r.queued)
        if n > 0:
            self.backend.enqueue(r.handle, n)
            r.queued += n

    def _sleep_until(self, t_target, now):
        dt = t_target - now()
        if dt > 0:
            time.sleep(min(dt, 0.01))

    @staticmethod
    def stats(runs, makespan, peak_bytes, max_concurrent):
        ok = [r for r in runs if r.error is None and r.done is not None]
        lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
        return {"completed": len(ok), "rejected": sum(1 for r in runs if r.error is not None),
                "makespan_s": makespan, "sims_per_s": len(ok) / makespan if makespan > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_mean_s": float(lat.mean()), "peak_resident_bytes": int(peak_bytes),
                "max_concurrent": int(max_concurrent)}


def make_runs(specs, backend):
    """Build each request's case and its device footprint (before the clock starts)."""
    runs = []
    for s in specs:
        case = s.case()
        runs.append(Run(s, case, backend.bytes_needed(case)))
    return runs
