"""Serving loop: request stream, HBM-budget admission, continuous batching, alone-vs-mix results.

The host logic (stream, admission, accounting, percentiles) runs on the CPU against a simulated
backend with a virtual clock; the GPU tests run real requests and compare each result with the
same request run alone.
"""
import numpy as np
import pytest

from epp import serve


# ---------------------------------------------------------------------------- host logic (CPU)

class TickClock:
    """Virtual clock that advances a fixed tick on every read."""

    def __init__(self, tick=1e-4):
        self.t = 0.0
        self.tick = tick

    def __call__(self):
        self.t += self.tick
        return self.t


class FakeCase:
    def __init__(self, n, key=None):
        self.n = n
        self.key = key


class FakeHandle:
    def __init__(self, case):
        self.case = case
        self.busy_until = 0.0


class FakeBackend:
    """A device that runs each resident simulation at `cost` seconds per particle-step, every
    resident run concurrently (streams), and records the admission order."""

    def __init__(self, clock, cost=1e-9):
        self.clock = clock
        self.cost = cost
        self.admitted = []

    def bytes_needed(self, case):
        return case.n * 1000

    def admit(self, case):
        self.admitted.append(case)
        h = FakeHandle(case)
        h.busy_until = self.clock.t
        return h

    def enqueue(self, h, n):
        h.busy_until = max(h.busy_until, self.clock.t) + n * h.case.n * self.cost

    def idle(self, h):
        return self.clock.t >= h.busy_until

    def finish(self, h):
        return {"n": h.case.n}

    def group_key(self, case):
        return case.key

    def admit_group(self, cases):
        self.admitted.append(tuple(c.n for c in cases))
        h = FakeHandle(FakeCase(sum(c.n for c in cases)))
        h.members = cases
        h.busy_until = self.clock.t
        return h

    def finish_group(self, h, k):
        assert k == len(h.members)
        return [{"n": c.n, "batch": len(h.members)} for c in h.members]


def fake_runs(sizes, arrivals, steps=100, keys=None):
    runs = []
    for i, (n, t) in enumerate(zip(sizes, arrivals)):
        st = steps[i] if isinstance(steps, list) else steps
        k = keys[i] if keys else None
        spec = serve.RequestSpec(i, t, 2, n, 1.0, st)
        runs.append(serve.Run(spec, FakeCase(n, k), n * 1000, k))
    return runs


def test_request_stream_is_seeded_and_shaped():
    a = serve.request_stream(2000, seed=3)
    b = serve.request_stream(2000, seed=3)
    assert [(r.arrival, r.dim, r.n_fluid, r.aspect) for r in a] == [(r.arrival, r.dim, r.n_fluid, r.aspect) for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert abs(np.mean(np.diff(arr)) - 1.0 / 50.0) < 0.1 / 50.0          # Poisson, mean 50 / s
    frac2 = np.mean([r.dim == 2 for r in a])
    assert 0.66 < frac2 < 0.74                                            # 70% 2D
    n = np.array([r.n_fluid for r in a])
    assert n.min() >= 1000 and n.max() <= 1000000
    assert abs(np.median(np.log10(n)) - 4.5) < 0.15                       # log-uniform 1e3 - 1e6
    asp = np.array([r.aspect for r in a])
    assert asp.min() >= 0.5 and asp.max() <= 2.5


def test_fifo_admission_within_budget():
    clock = TickClock()
    be = FakeBackend(clock)
    sizes = [5000, 40000, 2000, 30000, 8000, 60000, 1000, 20000]
    runs = fake_runs(sizes, [0.001 * i for i in range(len(sizes))])
    budget = 70000 * 1000
    st = serve.Server(be, budget_bytes=budget, clock=clock, idle_wait=0.0).run(runs)
    assert st["completed"] == len(sizes) and st["rejected"] == 0
    assert st["peak_resident_bytes"] <= budget
    assert [c.n for c in be.admitted] == sizes                            # FIFO order
    adm = [r.admitted for r in runs]
    assert adm == sorted(adm)
    assert st["max_concurrent"] >= 2                                      # runs overlap


def test_oversize_request_rejected_others_served():
    clock = TickClock()
    be = FakeBackend(clock)
    runs = fake_runs([1000, 10**6, 2000], [0.0, 0.001, 0.002])
    st = serve.Server(be, budget_bytes=5 * 10**6, clock=clock, idle_wait=0.0).run(runs)
    assert st["completed"] == 2 and st["rejected"] == 1
    assert runs[1].error and runs[1].result is None
    assert runs[0].result == {"n": 1000} and runs[2].result == {"n": 2000}


def test_one_at_a_time_is_sequential_and_slower():
    sizes = [20000, 5000, 50000, 10000, 30000]
    arr = [0.0, 0.0005, 0.001, 0.0015, 0.002]
    c1 = TickClock()
    seq = fake_runs(sizes, arr)
    st1 = serve.Server(FakeBackend(c1), max_active=1, clock=c1, idle_wait=0.0).run(seq)
    for a, b in zip(seq, seq[1:]):
        assert b.admitted >= a.done                                       # no overlap
    c2 = TickClock()
    mix = fake_runs(sizes, arr)
    st2 = serve.Server(FakeBackend(c2), clock=c2, idle_wait=0.0).run(mix)
    assert st2["makespan_s"] < st1["makespan_s"]
    assert st2["latency_p99_s"] < st1["latency_p99_s"]
    lat = sorted(r.latency for r in mix)
    assert abs(st2["latency_p50_s"] - float(np.percentile(lat, 50))) < 1e-12


def test_co_batching_groups_waiting_requests():
    """Waiting requests with equal keys and step counts are admitted as one batch (budget and
    max_active respected); others run alone; every member gets its own result."""
    clock = TickClock()
    be = FakeBackend(clock)
    sizes = [1000, 2000, 3000, 4000, 5000, 6000, 7000]
    keys = ["a", "a", "b", "a", None, "a", "a"]
    steps = [100, 100, 100, 100, 100, 50, 100]
    runs = fake_runs(sizes, [0.0] * len(sizes), steps=steps, keys=keys)
    st = serve.Server(be, clock=clock, idle_wait=0.0, co_batch=True).run(runs)
    assert st["completed"] == len(sizes)
    # the head "a" takes every waiting "a" with 100 steps; the 50-step "a" runs alone
    assert be.admitted[0] == (1000, 2000, 4000, 7000)
    assert [getattr(c, "n", c) for c in be.admitted[1:]] == [3000, 5000, 6000]
    for r in runs:
        assert r.result["n"] == r.spec.n_fluid
    grouped = [runs[i] for i in (0, 1, 3, 6)]
    assert len({r.done for r in grouped}) == 1 and all(r.result["batch"] == 4 for r in grouped)
    # a budget that holds two of them: the group stops growing at the budget
    clock2 = TickClock()
    be2 = FakeBackend(clock2)
    runs2 = fake_runs([1000, 1000, 1000], [0.0] * 3, keys=["a"] * 3)
    st2 = serve.Server(be2, budget_bytes=2000 * 1000, clock=clock2, idle_wait=0.0, co_batch=True).run(runs2)
    assert st2["completed"] == 3 and st2["peak_resident_bytes"] <= 2000 * 1000
    assert be2.admitted[0] == (1000, 1000)
    # without co-batching nothing is grouped
    clock3 = TickClock()
    be3 = FakeBackend(clock3)
    serve.Server(be3, clock=clock3, idle_wait=0.0).run(fake_runs([1000, 1000], [0.0, 0.0], keys=["a", "a"]))
    assert all(not isinstance(c, tuple) for c in be3.admitted)


# ---------------------------------------------------------------------------- device (GPU)

def _small_stream(n=6, steps=200, seed=1):
    return serve.request_stream(n, seed=seed, rate=500.0, n_range=(1e3, 2e4), steps=steps)


@pytest.mark.gpu
def test_served_results_equal_alone():
    specs = _small_stream()
    be = serve.DeviceBackend(download=True)
    runs = serve.make_runs(specs, be)
    st = serve.Server(be, chunk=50).run(runs)
    assert st["completed"] == len(specs)
    assert st["max_concurrent"] >= 2
    for r in runs:
        alone = serve.DeviceBackend(download=True)
        case = r.spec.case()
        h = alone.admit(case)
        alone.enqueue(h, r.spec.steps)
        res = alone.finish(h)
        assert r.result["status"] == res["status"]
        for k, v in res["state"].items():
            assert np.array_equal(r.result["state"][k], v), (r.spec.rid, k)
        for k in ("mass_total", "kinetic", "potential", "internal", "n_pairs"):
            assert r.result["integrals"][k] == res["integrals"][k], (r.spec.rid, k)


@pytest.mark.gpu
def test_budget_limits_resident_runs():
    specs = _small_stream(n=5, steps=100, seed=2)
    be = serve.DeviceBackend()
    runs = serve.make_runs(specs, be)
    budget = max(r.bytes for r in runs) + min(r.bytes for r in runs) // 2
    st = serve.Server(be, budget_bytes=budget, chunk=50).run(runs)
    assert st["completed"] == len(specs) and st["rejected"] == 0
    assert st["peak_resident_bytes"] <= budget


@pytest.mark.gpu
def test_co_batched_results_equal_alone():
    """Requests of the 256-instance mix served co-batched (one batch context) give each
    instance's state bit-identical to that request run alone; its FP64 integrals agree to the
    rounding of the per-instance reduction order (1e-12)."""
    specs = serve.batch_mix_requests(6, steps=60)
    be = serve.DeviceBackend(download=True)
    runs = serve.make_runs(specs, be)
    assert len({r.group_key for r in runs}) == 1
    st = serve.Server(be, chunk=20, co_batch=True).run(runs)
    assert st["completed"] == len(specs)
    assert len({r.done for r in runs}) == 1          # one batch
    for r in runs:
        alone = serve.DeviceBackend(download=True)
        h = alone.admit(r.spec.case())
        alone.enqueue(h, r.spec.steps)
        res = alone.finish(h)
        for k, v in res["state"].items():
            assert np.array_equal(r.result["state"][k], v), (r.spec.rid, k)
        assert r.result["integrals"]["n_pairs"] == res["integrals"]["n_pairs"]
        for k in ("mass_total", "kinetic", "potential", "internal"):
            assert abs(r.result["integrals"][k] - res["integrals"][k]) <= 1e-12 * abs(res["integrals"][k]), (r.spec.rid, k)


# ---------------------------------------------------------------------------- native loop (C ABI)

def test_native_server_argument_checks():
    """epp_server_create validates its arguments before touching a device, and without a GPU it
    fails loudly (no CPU fallback)."""
    import ctypes as C

    from epp import abi, lib as epplib
    lib = epplib.load()
    h = C.c_void_p()
    assert lib.epp_server_create(0, 0, 4, 100, 2, C.byref(h)) == abi.EPP_ERR_INVALID_ARGUMENT
    assert lib.epp_server_create(0, 10**9, 0, 100, 2, C.byref(h)) == abi.EPP_ERR_INVALID_ARGUMENT
    n = C.c_int32(0)
    if lib.epp_device_count(C.byref(n)) != abi.EPP_OK:
        with pytest.raises(epplib.EppError) as e:
            epplib.NativeServer()
        assert e.value.code == abi.EPP_ERR_NO_DEVICE


def _native_submit(srv, specs, steps, keep_state=True):
    be = serve.DeviceBackend()
    cases, ids = [], []
    for s in specs:
        c = s.case()
        _, cfg = be.config_of(c)
        cases.append(c)
        ids.append(srv.submit(cfg, c.ps, c.ps.column_map(), c.physics, steps, keep_state=keep_state))
    return cases, ids


@pytest.mark.gpu
def test_native_server_results_equal_alone():
    """The C-ABI serving loop: every request's integrals and final state equal the same
    simulation run alone, with several requests resident at once."""
    from epp.lib import EppError, NativeServer
    from epp import abi
    steps = 120
    specs = _small_stream(n=5, steps=steps, seed=4)
    srv = NativeServer(chunk_steps=50)
    cases, ids = _native_submit(srv, specs, steps)
    with pytest.raises(EppError) as e:   # not finished yet: nothing has run before a poll
        srv.result(ids[0])
    assert e.value.code == abi.EPP_ERR_STATE
    st = srv.drain()
    assert st["completed"] == len(specs) and st["failed"] == 0 and st["max_concurrent"] >= 2
    for spec, rid in zip(specs, ids):
        res = srv.result(rid)
        assert 0 <= res["admit_s"] <= res["done_s"]
        alone = serve.DeviceBackend(download=True)
        h = alone.admit(spec.case())
        alone.enqueue(h, steps)
        ref = alone.finish(h)
        assert res["status"] == ref["status"]
        for k in ("mass_total", "kinetic", "potential", "internal", "n_pairs", "n_alive"):
            assert res["integrals"][k] == ref["integrals"][k], (spec.rid, k)
        out = spec.case()
        srv.download(rid, out.ps)
        for k, v in ref["state"].items():
            assert np.array_equal(out.ps[k], v), (spec.rid, k)
    srv.close()


@pytest.mark.gpu
def test_native_server_budget():
    """Resident bytes stay within the budget; a request that can never fit fails with
    EPP_ERR_BUDGET while the others are served."""
    from epp.lib import EppError, NativeServer, context_bytes
    from epp import abi
    steps = 40
    specs = _small_stream(n=4, steps=steps, seed=5)
    be = serve.DeviceBackend()
    sizes = [context_bytes(be.config_of(s.case())[1]) for s in specs]
    budget = max(sizes) + min(sizes) // 2
    srv = NativeServer(budget_bytes=budget, chunk_steps=20)
    cases, ids = _native_submit(srv, specs, steps, keep_state=False)
    st = srv.drain()
    assert st["completed"] == len(specs) and st["peak_resident_bytes"] <= budget
    srv.close()
    small = NativeServer(budget_bytes=min(sizes) // 2, chunk_steps=20)
    _, ids = _native_submit(small, specs[:2], steps, keep_state=False)
    st = small.drain()
    assert st["failed"] == 2 and st["completed"] == 0
    with pytest.raises(EppError) as e:
        small.result(ids[0])
    assert e.value.code == abi.EPP_ERR_BUDGET
    small.close()


@pytest.mark.gpu
def test_native_server_co_batching_equals_alone():
    """Co-batching in the C-ABI loop: requests of the 256-instance mix waiting together become one
    batch context; each request's state is bit-identical to the request run alone, its FP64
    integrals equal to the rounding of the per-instance reduction order (1e-12)."""
    from epp.lib import NativeServer
    steps = 60
    specs = serve.batch_mix_requests(5, steps=steps)
    srv = NativeServer(chunk_steps=20, co_batch=True)
    cases, ids = _native_submit(srv, specs, steps)
    st = srv.drain()
    assert st["completed"] == len(specs) and st["failed"] == 0
    assert st["max_concurrent"] == len(specs)   # all five resident together, as one batch
    for spec, rid in zip(specs, ids):
        res = srv.result(rid)
        alone = serve.DeviceBackend(download=True)
        h = alone.admit(spec.case())
        alone.enqueue(h, steps)
        ref = alone.finish(h)
        assert res["integrals"]["n_pairs"] == ref["integrals"]["n_pairs"]
        for k in ("mass_total", "kinetic", "potential", "internal"):
            assert abs(res["integrals"][k] - ref["integrals"][k]) <= 1e-12 * abs(ref["integrals"][k]), (spec.rid, k)
        out = spec.case()
        srv.download(rid, out.ps)
        for k, v in ref["state"].items():
            assert np.array_equal(out.ps[k], v), (spec.rid, k)
    srv.close()
