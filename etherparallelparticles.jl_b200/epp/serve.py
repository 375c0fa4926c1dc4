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
the same whether it runs alone or in the mix.  With co-batching, requests that wait together and
can share a cell grid and physics (2D, same tank and lattice spacing, same step count; dt and c0
may differ) are admitted as the instances of one batch context, so their steps run as one launch
per pass; an instance gives the same bits in a batch as alone.

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

    def __init__(self, spec, case, nbytes, group_key=None):
        self.spec = spec
        self.case = case
        self.bytes = nbytes
        self.group_key = group_key   # equal keys (and step counts) may share one batch context
        self.handle = None
        self.queued = 0          # steps enqueued on the device
        self.admitted = None     # seconds after start
        self.done = None
        self.result = None
        self.error = None
        self.runs = [self]       # the requests this resident unit serves

    @property
    def steps(self):
        return self.spec.steps

    @property
    def latency(self):
        return None if self.done is None else self.done - self.spec.arrival


class Group:
    """Requests co-batched into one batch context: resident, stepped and retired together."""

    def __init__(self, runs):
        self.runs = runs
        self.bytes = sum(r.bytes for r in runs)   # a batch needs at most its instances' sum
        self.handle = None
        self.queued = 0

    @property
    def steps(self):
        return self.runs[0].spec.steps


class DeviceBackend:
    """Runs each request on its own epp context (own stream) on one GPU."""

    def __init__(self, device=0, download=False, priorities=True, tuner=None, tune_concurrent=True):
        self.device = device
        self.download = download
        self.priorities = priorities
        self.tuner = tuner        # autotune.Autotuner: launch configuration per dimension and size
        self.tune_concurrent = tune_concurrent   # tune for throughput with several runs resident

    def config_of(self, case):
        """(NeighbourSystem, epp_config) of a request's case on this backend's device."""
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
        return context_bytes(self.config_of(case)[1])

    def admit(self, case):
        from .algorithm import DeviceParticleSystem
        ns, _ = self.config_of(case)
        dps = DeviceParticleSystem(case.ps, ns, device=self.device)
        dps.physics = case.physics
        if self.priorities:
            dps.ctx.set_priority(priority_for(case.n))
        if self.tuner is not None:
            self.tuner.apply(dps.ctx, case.meta["dim"], case.n, concurrent=self.copies(case.n))
        dps.syncto()
        dps.ctx.search(SYM, CONT, case.physics, 0)
        return dps

    def group_key(self, case):
        return casegen.batch_key(case)

    def admit_group(self, cases):
        """One batch context holding `cases` as instances 0..K-1 (casegen.merge_cases)."""
        from .algorithm import DeviceParticleSystem
        b = casegen.merge_cases(cases)
        ns, _ = self.config_of(b)
        dps = DeviceParticleSystem(b.ps, ns, device=self.device, n_instances=b.n_instances)
        dps.physics = b.physics
        dps.batch = b
        dps.ctx.set_instance_physics(b.inst_dt, b.inst_c0)
        if self.priorities:
            dps.ctx.set_priority(priority_for(b.n))
        best = self.tuner.cached(2, b.n, batch=True) if self.tuner is not None else None
        if best is not None:   # batches run family 0; a block size is used only if already tuned
            dps.ctx.set_block_threads(best[1])
        dps.syncto()
        dps.ctx.search(SYM, CONT, b.physics, 0)
        return dps

    def finish_group(self, dps, k):
        st = dps.ctx.synchronize(raise_on_status=False)
        integ = dps.ctx.instance_integrals(dps.physics, k)
        out = [{"integrals": integ[i], "status": st} for i in range(k)]
        if self.download:
            dps.asyncto()
            h = dps.host
            for i, (a, e) in enumerate(dps.batch.rows):
                out[i]["state"] = {c: h[c][a:e] for c in ("PositionVec", "VelocityVec", "Density", "Pressure", "nCount")}
        dps.close()
        return out

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
                 clock=time.perf_counter, idle_wait=50e-6, co_batch=False, batch_max=256):
        self.backend = backend
        self.co_batch = co_batch      # admit waiting requests with equal group keys as one batch
        self.batch_max = batch_max
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
        active = []              # resident units: Run, or Group of co-batched runs
        used = peak = 0
        max_conc = 0
        n_res = 0                # resident requests
        while arrivals or waiting or active:
            t = now()
            while arrivals and arrivals[0].spec.arrival <= t:
                waiting.append(arrivals.popleft())
            # FIFO admission while the head fits the budget and a slot is free
            while waiting and n_res < self.max_active:
                r = waiting[0]
                if r.bytes > self.budget:          # can never fit: reject, keep serving the rest
                    waiting.popleft()
                    r.error = "needs %d bytes, budget %d" % (r.bytes, self.budget)
                    r.done = now()
                    continue
                if used + r.bytes > self.budget:
                    break
                waiting.popleft()
                members = [r]
                if self.co_batch and r.group_key is not None:
                    # the waiting requests that can share the head's batch, in arrival order
                    room = self.budget - used - r.bytes
                    for w in list(waiting):
                        if len(members) >= min(self.batch_max, self.max_active - n_res):
                            break
                        if w.group_key == r.group_key and w.spec.steps == r.spec.steps and w.bytes <= room:
                            members.append(w)
                            waiting.remove(w)
                            room -= w.bytes
                if len(members) == 1:
                    unit = r
                    r.handle = self.backend.admit(r.case)
                else:
                    unit = Group(members)
                    unit.handle = self.backend.admit_group([m.case for m in members])
                t_adm = now()
                for m in members:
                    m.admitted = t_adm
                used += unit.bytes
                peak = max(peak, used)
                n_res += len(members)
                active.append(unit)
                self._fill(unit)
            max_conc = max(max_conc, n_res)
            progressed = False
            for r in list(active):
                if not self.backend.idle(r.handle):
                    continue
                progressed = True
                if r.queued < r.steps:
                    self._fill(r)
                    continue
                if isinstance(r, Group):
                    results = self.backend.finish_group(r.handle, len(r.runs))
                else:
                    results = [self.backend.finish(r.handle)]
                t_done = now()
                for m, res in zip(r.runs, results):
                    m.result = res
                    m.done = t_done
                r.handle = None
                used -= r.bytes
                n_res -= len(r.runs)
                active.remove(r)
            if not progressed:
                if not active and not waiting and arrivals:
                    self._sleep_until(arrivals[0].spec.arrival, now)
                else:
                    time.sleep(self.idle_wait)
        makespan = now()
        return self.stats(runs, makespan, peak, max_conc)

    def _fill(self, r):
        n = min(self.chunk * self.ahead, r.steps - r.queued)
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
    """Build each request's case, its device footprint and its batch key (before the clock
    starts)."""
    runs = []
    for s in specs:
        case = s.case()
        key = backend.group_key(case) if hasattr(backend, "group_key") else None
        runs.append(Run(s, case, backend.bytes_needed(case), key))
    return runs


def serve_native(specs, device=0, budget_bytes=120 * 10**9, max_active=256, chunk=100, ahead=2,
                 clock=time.perf_counter, idle_wait=50e-6, co_batch=False):
    """The same request trace through the native serving loop (epp_server_*, the C ABI): each
    request is submitted when its arrival time passes (its case built beforehand), the loop is
    polled in between; returns the stats of Server.run (latency = completion - arrival)."""
    from .lib import EppError, NativeServer
    be = DeviceBackend(device=device)
    prepared = []
    for s in specs:
        c = s.case()
        prepared.append((s, c, be.config_of(c)[1], c.ps.column_map()))
    srv = NativeServer(device=device, budget_bytes=budget_bytes, max_active=max_active, chunk_steps=chunk,
                       ahead=ahead, co_batch=co_batch)
    order = collections.deque(sorted(prepared, key=lambda p: p[0].arrival))
    ids = {}
    t0 = clock()
    st = {}
    while order or not st or st["waiting"] or st["active"]:
        t = clock() - t0
        while order and order[0][0].arrival <= t:
            s, c, cfg, cmap = order.popleft()
            ids[s.rid] = (s, srv.submit(cfg, c.ps, cmap, c.physics, s.steps))
        st = srv.poll()
        if not order and not st["waiting"] and not st["active"]:
            break
        time.sleep(idle_wait)
    makespan = clock() - t0
    lat, done = [], 0
    for s, rid in ids.values():
        try:
            r = srv.result(rid)
        except EppError:
            continue
        done += 1
        lat.append(r["done_s"])   # submitted when its arrival time passed: completion - arrival
    lat = np.array(lat) if lat else np.zeros(1)
    out = {"completed": done, "rejected": int(st.get("failed", 0)), "makespan_s": makespan,
           "sims_per_s": done / makespan if makespan > 0 else 0.0,
           "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
           "latency_mean_s": float(lat.mean()), "peak_resident_bytes": int(st.get("peak_resident_bytes", 0)),
           "max_concurrent": int(st.get("max_concurrent", 0)), "loop": "native (epp_server_*)",
           "latencies": [float(x) for x in lat]}
    srv.close()
    return out
