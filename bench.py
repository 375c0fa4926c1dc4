"""Benchmark of the SPH time step (pair-interactions/s) on B200.

Default workload (N=1): the 2D dam break at dx = 0.002 m -- 500,000 fluid particles plus the
3-layer walls (15,018 particles), cell gap 2h, re-sorted every step, Wendland C2, Tait EOS,
artificial viscosity, symplectic Euler with Kahan positions.  A step is one full time step of
example/collapse_dry/same/main.jl:166-182 (density update, momentum, integrate, search +
continuity).  The metric counts the directed active neighbour pairs of each step's search once.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl epp|reference] [--case 2d|3d|2d-small|3d-small]

N > 1 (torchrun): the plain path does not shard, so every rank runs an independent replica
("replicas only"), no collective on the data path; value = pairs of all ranks / max time.

--impl reference times the CPU restatement of the reference algorithm (the oracle: stored
neighbour lists, bucket cell list, one pass per reference launch) on the host cores.
"""
import argparse
import json
import os
import re
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "etherparallelparticles.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

# Algorithmic bytes per particle per step: the compulsory traffic of a step in which each
# particle's record is read and written once and neighbour data is served on chip (stage table):
#   momentum pass      read x, v, rho, drho, id, Kahan c; write x, c, v, rho       2D 64,  3D 88
#   hash + count       read x; write cell key; histogram atomic                    2D 16,  3D 20
#   scan               8 B per cell, per particle                                  2D 5,   3D 0.5
#   scatter / reorder  read key + rank; gather state; write sorted state           2D 80,  3D 104
#   continuity         read x, v, id; write drho                                   2D 24,  3D 32
#   whole step                                                                     2D 189, 3D 245
# The six kernels of a step re-split those stages: the momentum pass also bins (momentum + hash
# and count), the reorder is the scatter (key + rank, 8 B) and the rank-by-id gather (the rest),
# and the continuity stage is split between the search pass (reads x and id) and the continuity
# pass (reads v, writes drho).  The per-kernel figures add up to the whole step.
B_ALG_STEP = {2: 189.0, 3: 245.0}
STAGES = ["momentum_integrate_bin", "scan", "scatter", "rank_gather", "search", "continuity"]
B_ALG_STAGE = {"momentum_integrate_bin": {2: 80.0, 3: 108.0}, "scan": {2: 5.0, 3: 0.5},
               "scatter": {2: 8.0, 3: 8.0}, "rank_gather": {2: 72.0, 3: 96.0},
               "search": {2: 12.0, 3: 16.0}, "continuity": {2: 12.0, 3: 16.0}}
PAIR_STAGES = ("momentum_integrate_bin", "search", "continuity")
KERNEL_OF_STAGE = {"momentum_integrate_bin": "k_list<CPMom> (momentum + integrate + bin, fused)",
                   "scan": "k_scan (decoupled look-back exclusive scan)",
                   "scatter": "k_scatter (arrival-order scatter)",
                   "rank_gather": "k_rank_gather (rank by id + state gather + density update)",
                   "search": "k_build (neighbour lists + nCount)",
                   "continuity": "k_list<CPCont> (continuity + density preview, fused)"}


def kernel_key(name):
    """(kernel, first type argument) of a kernel label or an ncu kernel name:
    "k_list<CPMom> (...)" and "k_list<2, CPMom<2, 1, 0>, 1>" both give ("k_list", "CPMom")."""
    head = name.split(" (")[0]
    m = re.search(r"[<,]\s*([A-Za-z_]\w*)", head)
    return head.split("<")[0], m.group(1) if m else None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="epp", choices=["epp", "reference"])
    ap.add_argument("--case", default="2d", choices=["2d", "3d", "2d-small", "3d-small", "batch", "serve"])
    ap.add_argument("--instances", type=int, default=256, help="batch: number of instances")
    ap.add_argument("--requests", type=int, default=32, help="serve: number of requests in the stream")
    ap.add_argument("--sim-steps", type=int, default=2000, help="serve: steps per request")
    ap.add_argument("--native", action="store_true",
                    help="serve: run the trace through the native serving loop of the C ABI (epp_server_*)")
    ap.add_argument("--no-co-batch", dest="co_batch", action="store_false",
                    help="serve: give every request its own context (no co-batching of waiting requests)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="batch / serve: skip the launch-configuration autotuner (serve)")
    ap.add_argument("--mix", default="stream", choices=["stream", "batch"],
                    help="serve: the Poisson request stream, or the batched form's 256-instance mix as a burst")
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--physics", default="benchmark", choices=["benchmark", "example"],
                    help="2D cases: the benchmark physics, or the reference example's own (CubicSpline, "
                         "linear EOS, classic viscosity, sAccelerateMove!, kernel filter every 20 steps)")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per particle (0 = tuned default)")
    ap.add_argument("--no-served", dest="served", action="store_false",
                    help="2D line: skip the batch and serve legs (batched and served sims/s)")
    ap.add_argument("--no-parity", dest="parity", action="store_false",
                    help="skip the untimed parity check of the workload against the oracle")
    ap.add_argument("--leg-requests", type=int, default=16,
                    help="2D line's serve leg: requests of the Poisson stream served (the first ones)")
    return ap.parse_args()


def plain_config(case, label, world, flush=True):
    """The workload keys of the plain-path line (the same in both arms)."""
    m = case.meta
    return {"workload": label, "particles": case.n, "fluid": m["n_fluid"], "walls": m["n_wall"],
            "cells": m["n_cells"], "resort": "every step",
            "l2": "flushed (256 MB write) before every timed step" if flush else "not flushed",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def make_case(name, physics="benchmark"):
    from epp import casegen
    tag = "" if physics == "benchmark" else ", example physics"
    if name == "2d":
        return (casegen.dam_break_2d(dx=0.002, max_neighbour_number=1, physics=physics),
                "2D dam break dx=0.002 (500k fluid%s)" % tag)
    if name == "2d-small":
        return (casegen.dam_break_2d(dx=0.02, max_neighbour_number=1, physics=physics),
                "2D dam break dx=0.02 (5k fluid%s)" % tag)
    if name == "3d-small":
        return casegen.dam_break_3d(dx=0.01, max_neighbour_number=1), "3D dam break dx=0.01 (600k fluid)"
    return casegen.dam_break_3d(dx=0.005, max_neighbour_number=1), "3D dam break dx=0.005 (4.8M fluid)"


class Clocks:
    """SM clock and clock-event reasons, polled through NVML (read-only queries) every ~2 ms
    from a host thread while the timed region runs."""

    REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown")]

    def __init__(self, torch_device):
        self.dev = torch_device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.stop_flag = threading.Event()
        self.t = None
        self.nv = None
        self.h = None

    def _handle(self):
        import pynvml as nv
        import torch
        nv.nvmlInit()
        pr = torch.cuda.get_device_properties(self.dev)
        bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        self.nv = nv
        self.h = nv.nvmlDeviceGetHandleByPciBusId(bus)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))

    def start(self):
        try:
            self._handle()
        except Exception:
            self.h = None
            return
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def _poll(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_flag.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                bits = get_reasons(self.h)
                for name, const in self.REASONS:
                    if bits & getattr(nv, const, 0):
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def stop(self):
        if self.t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        self.stop_flag.set()
        self.t.join(timeout=5)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml, 2 ms poll"}


def cpu_reference(case, steps_budget_s=20.0, max_steps=3, warmup=0):
    """The oracle (C++ restatement of the reference's CPU algorithm) on all host cores, after
    `warmup` untimed steps."""
    from epp import abi
    from epp.classes import NeighbourSystem
    from epp import casegen
    import oracle_lib
    ps, phys = case.ps, case.physics
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40 if case.meta["dim"] == 2 else 100)
    cfg = abi.make_config(case.domain.to_abi(), ps.n_capacity, ns.active_pair.adjacency_matrix.tolist(),
                          max_neighbour_number=ns.max_neighbour_number, max_cell_particles=64 if case.meta["dim"] == 2 else 128)
    threads = os.cpu_count() or 1
    oracle_lib.set_threads(threads)
    o = oracle_lib.Oracle(cfg, 32)
    o.lib.orc_set_deterministic(o.h, 0)   # threaded atomic insert, as the reference's CPU backend
    cm = ps.column_map()
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, cm)
    o.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY, phys)
    if warmup:
        o.step(warmup, phys)
    pairs, t_total, steps = 0, 0.0, 0
    while steps < max_steps and (steps == 0 or t_total < steps_budget_s):
        t0 = time.perf_counter()
        o.step(1, phys)
        t_total += time.perf_counter() - t0
        pairs += int(o.field(9, 0, ps.n_particles).sum())
        steps += 1
    return {"value": pairs / t_total, "unit": "pair-interactions/s", "cores": threads, "kind": "port",
            "pairs_per_step": pairs / steps,
            "sample": "%d full steps of %s (%d particles), %.2f s" % (steps, case.meta.get("label", ""), ps.n_particles, t_total),
            "seconds_per_step": t_total / steps}


def run_reference(args):
    """--impl reference: the CPU restatement on the host cores, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.case == "batch":
        return run_reference_batch(args)
    if args.case == "serve":
        return run_reference_serve(args)
    case, label = make_case(args.case, args.physics)
    case.meta["label"] = label
    probe = cpu_reference(case, steps_budget_s=0.0, max_steps=1)      # cost of one step
    k = max(1, min(args.steps, int(120.0 / max(probe["seconds_per_step"], 1e-3))))
    w = max(0, min(args.warmup, int(30.0 / max(probe["seconds_per_step"], 1e-3))))
    res = cpu_reference(case, steps_budget_s=150.0, max_steps=k, warmup=w)
    val = res["value"]
    out = {"metric": "SPH pair-interactions/s", "value": val, "unit": "pair-interactions/s",
           "impl": "reference", "n_gpus": args.gpus, "steps": k, "warmup": w,
           "ms_per_step": res["seconds_per_step"] * 1e3, "pairs_per_step": res["pairs_per_step"],
           "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (dam-break lattice generated in-process)",
           "config": plain_config(case, label, args.gpus, not args.no_flush),
           "cpu_baseline": {"value": val, "unit": "pair-interactions/s", "cores": res["cores"],
                            "kind": "port", "sample": res["sample"]},
           "e2e": {"value": val, "unit": "pair-interactions/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference_batch(args):
    """--impl reference --case batch: the oracle runs simulations one at a time (the reference has
    no batched form); sims/s from the mean step time of every 16th instance of the mix."""
    from epp import casegen
    cols = casegen.batch_columns(args.instances, seed=0)
    sample = list(range(0, len(cols), 16))
    per_step, cores, n_p = [], 1, 0
    for k in sample:
        case = casegen.dam_break_2d(dx=0.01, column=cols[k], max_neighbour_number=1)
        case.meta["label"] = "instance %d" % k
        res = cpu_reference(case, steps_budget_s=1.0, max_steps=max(1, min(args.steps, 10)))
        per_step.append(res["seconds_per_step"])
        cores = res["cores"]
        n_p += case.n
    val = 1.0 / (2000 * float(np.mean(per_step)))
    sample_txt = "instances %s of the %d-instance mix (%d particles), mean %.2f ms/step" % (
        sample, len(cols), n_p, 1e3 * float(np.mean(per_step)))
    out = {"metric": "batched sims/s (256-instance 2D dam-break mix, 2000 steps per simulation)",
           "value": val, "unit": "sims/s", "impl": "reference", "n_gpus": args.gpus,
           "steps": max(1, min(args.steps, 10)), "warmup": 0, "ms_per_step": 1e3 * float(np.mean(per_step)),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded column sizes, numpy default_rng(0))",
           "config": {"workload": "%d uneven 2D dam breaks, dx=0.01 m" % len(cols), "instances": len(cols)},
           "cpu_baseline": {"value": val, "unit": "sims/s", "cores": cores, "kind": "port", "sample": sample_txt},
           "e2e": {"value": val, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference_serve(args):
    """--impl reference --case serve: the oracle serves requests one at a time (the reference has
    no serving form); sims/s from a sample of the stream's requests timed for a few steps each."""
    from epp import serve
    specs = serve.request_stream(args.requests, seed=0, steps=args.sim_steps)
    sample = specs[:: max(1, len(specs) // 6)]
    total, cores = 0.0, 1
    for s in sample:
        case = s.case()
        case.meta["label"] = "request %d" % s.rid
        res = cpu_reference(case, steps_budget_s=2.0, max_steps=5)
        total += res["seconds_per_step"] * s.steps
        cores = res["cores"]
    val = len(sample) / total
    out = {"metric": "served sims/s (Poisson request stream, %d steps per simulation)" % args.sim_steps,
           "value": val, "unit": "sims/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.sim_steps,
           "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic request stream (numpy default_rng(0))",
           "config": {"workload": "%d requests" % args.requests},
           "cpu_baseline": {"value": val, "unit": "sims/s", "cores": cores, "kind": "port",
                            "sample": "requests %s, up to 5 steps each, one at a time" % [s.rid for s in sample]},
           "e2e": {"value": val, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def energy(ig):
    return ig["kinetic"] + ig["potential"] + ig["internal"]


def run_batch(args):
    """--case batch: the 256-instance mix of uneven 2D dam breaks (column width U[0.5, 1.5] m,
    height U[1.0, 2.5] m, seed 0, dx = 0.01 m, each instance with its own c0 and dt), every pass
    one launch over all instances.  value = sims/s at 2000 steps per simulation, against the
    plain path running the same instances one at a time (each timed alone on the device)."""
    import torch
    import torch.distributed as dist
    from epp import abi, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem
    import oracle_lib
    from helpers import config_for

    SIM_STEPS = 2000
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
    b = casegen.dam_break_batch(args.instances, seed=0, dx=0.01)
    phys = b.physics
    ns = NeighbourSystem(b.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    from epp import autotune
    tuned, tune_ms = autotune.tune_case(b, n_instances=b.n_instances, inst=(b.inst_dt, b.inst_c0), steps=5,
                                        device=local)
    dps = DeviceParticleSystem(b.ps, ns, device=local, n_instances=b.n_instances)
    ctx = dps.ctx
    ctx.set_instance_physics(b.inst_dt, b.inst_c0)
    ctx.set_block_threads(tuned[1])
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dps.syncto()
    ctx.search(SYM, CONT, phys, 0)
    e0 = [energy(x) for x in ctx.instance_integrals(phys, b.n_instances)]
    W = max(args.warmup, 3)
    with torch.cuda.stream(stream):
        ctx.step(W, phys)
    ctx.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = Clocks(local)
    p0 = ctx.pairs_total()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            ctx.step(1, phys)
            ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = ctx.synchronize(raise_on_status=False)
    ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
    pairs = ctx.pairs_total() - p0
    e1 = [energy(x) for x in ctx.instance_integrals(phys, b.n_instances)]
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
    step_ms = ms / args.steps
    sims_s = world * b.n_instances / (SIM_STEPS * step_ms * 1e-3)
    with torch.cuda.stream(stream):
        stage = np.mean([ctx.profile_step(phys) for _ in range(3)], axis=0)
    # end to end through the C ABI with pinned host buffers (upload, search, K x (step +
    # per-instance integrals read back), download)
    h = dps.host
    ip = np.asfortranarray(torch.from_numpy(np.asfortranarray(h.int_properties)).pin_memory().numpy())
    fp = np.asfortranarray(torch.from_numpy(np.asfortranarray(h.float_properties)).pin_memory().numpy())
    alive = torch.from_numpy(h.is_alive.copy()).pin_memory().numpy()
    cell = torch.from_numpy(h.cell_index.copy()).pin_memory().numpy()
    ctx.download(alive, cell, ip, fp, dps.cmap)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.upload(h.n_particles, alive, cell, ip, fp, dps.cmap)
    ctx.search(SYM, CONT, phys, 0)
    for _ in range(args.steps):
        ctx.step(1, phys)
        ctx.instance_integrals(phys, b.n_instances)
    ctx.download(alive, cell, ip, fp, dps.cmap)
    t_e2e = time.perf_counter() - t0
    n_cols = 2 * 3 + 6 + 5   # float columns moved (x, v, dv, m, V, rho, drho, p, h) + int (tag, mov, ncount, alive, cell, instance)
    bytes_io = h.n_particles * 4 * (n_cols + 1)
    dps.close()
    out = None
    if rank == 0:
        # plain path: every instance alone, one after the other, on one context sized for the
        # largest (the state of one instance stays resident in L2 between its own steps)
        K2 = 20
        cases = [casegen.dam_break_2d(dx=0.01, column=col, max_neighbour_number=1) for col in b.meta["columns"]]
        big = max(cases, key=lambda c: c.n)
        ns1 = NeighbourSystem(big.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        plain = DeviceParticleSystem(big.ps, ns1, device=local)
        pctx = plain.ctx
        pctx.set_stream(stream.cuda_stream)
        per_step = []
        for c in cases:
            q = c.ps
            pctx.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, plain.cmap)
            pctx.search(SYM, CONT, c.physics, 0)
            with torch.cuda.stream(stream):
                pctx.step(3, c.physics)
            torch.cuda.synchronize()
            a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                a_.record(stream)
                pctx.step(K2, c.physics)
                b_.record(stream)
            torch.cuda.synchronize()
            per_step.append(a_.elapsed_time(b_) / K2)
        plain.close()
        plain_sims_s = len(cases) / (SIM_STEPS * sum(per_step) * 1e-3)
        # energy drift against the FP64 oracle for sampled instances (the smallest three and the
        # largest), same number of steps from the same initial state
        S = W + args.steps
        order = sorted(range(len(cases)), key=lambda k: cases[k].n)
        sample = order[:3] + order[-1:]
        drift = {}
        oracle_lib.set_threads(os.cpu_count() or 1)
        for k in sample:
            c = casegen.dam_break_2d(dx=0.01, column=b.meta["columns"][k], max_neighbour_number=60)
            nso = NeighbourSystem(c.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=60)
            o = oracle_lib.Oracle(config_for(c.ps, nso, max_cell_particles=64), 64)
            q = c.ps
            o.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, q.column_map())
            o.search(SYM, CONT, c.physics)
            o0 = energy(o.integrals(c.physics))
            o.step(S, c.physics)
            o1 = energy(o.integrals(c.physics))
            dg, do = (e1[k] - e0[k]) / abs(e0[k]), (o1 - o0) / abs(o0)
            drift[str(k)] = {"particles": c.n, "gpu_fp32": dg, "oracle_fp64": do, "abs_diff": abs(dg - do)}
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except Exception:
            pass
        out = {
            "metric": "batched sims/s (256-instance 2D dam-break mix, 2000 steps per simulation)",
            "value": sims_s, "unit": "sims/s", "n_gpus": world, "steps": args.steps, "warmup": W,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded column sizes, numpy default_rng(0))",
            "config": {"workload": "%d uneven 2D dam breaks, width U[0.5,1.5] m, height U[1.0,2.5] m, dx=0.01 m"
                       % b.n_instances, "instances": b.n_instances, "particles": b.n,
                       "fluid": b.meta["n_fluid"], "walls": b.meta["n_wall"],
                       "fluid_per_instance": [min(b.meta["inst_n_fluid"]), max(b.meta["inst_n_fluid"])],
                       "cells": b.meta["n_cells"], "resort": "every step",
                       "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": "instances per GPU, replicas across GPUs" if world > 1 else "single GPU"},
            "plain_path": {"sims_per_s": plain_sims_s, "ms_per_instance_step_mean": float(np.mean(per_step)),
                           "ms_per_instance_step_range": [float(min(per_step)), float(max(per_step))],
                           "method": "each instance alone on the plain path (epp_step graph), %d steps "
                                     "timed per instance by CUDA events, summed over the %d instances"
                                     % (K2, len(cases))},
            "speedup_vs_plain": sims_s / world / plain_sims_s,
            "autotune": {"family": tuned[0], "block_threads": tuned[1], "resort_every": 1,
                         "ms_per_step": {"%d/%d" % k: round(v, 4) for k, v in tune_ms.items()}},
            "pairs_per_s": pairs / (ms * 1e-3) if world == 1 else None,
            "energy_drift": {"steps": S, "bar": 1e-4, "instances": drift,
                             "max_abs_diff": max(v["abs_diff"] for v in drift.values())},
            "gpu_launches": 5 * args.steps,
            "roofline": {"bound": "hbm", "stage_ms": dict(zip(STAGES, [round(float(x), 4) for x in stage])),
                         "achieved": B_ALG_STEP[2] * b.n / (step_ms * 1e-3) / 1e9,
                         "peak": peaks.get("hbm_gbs", 6650.0), "unit": "GB/s",
                         "frac": B_ALG_STEP[2] * b.n / (step_ms * 1e-3) / 1e9 / peaks.get("hbm_gbs", 6650.0),
                         "traffic": None, "note": "whole step, algorithmic bytes; pair kernels are issue/latency bound"},
            "clocks": clk,
            "e2e": {"value": b.n_instances * args.steps / SIM_STEPS / t_e2e, "unit": "sims/s",
                    "h2d_bytes_per_step": int(bytes_io / args.steps), "d2h_bytes_per_step": int(bytes_io / args.steps + 72 * b.n_instances),
                    "seconds": t_e2e,
                    "note": "upload + search + K x (step + per-instance integrals read back) + download, host clock"},
            "device_status": st,
        }
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_serve(args):
    """--case serve: the seeded request stream (Poisson arrivals, mean 50 / s; 70% 2D, 30% 3D; fluid
    counts log-uniform in 1e3 - 1e6; 2000 steps each) served under a 120 GB HBM budget per GPU with
    continuous batching, against the same trace served one request at a time on the plain path.
    value = completed simulations / makespan (arrival of the first request to completion of the
    last), latency = completion - arrival, both on the host clock; every request is uploaded,
    searched, stepped and read back (FP64 integrals) inside the measured time.  On N GPUs the
    stream is split by expected work (epp.ranks.partition) and every rank serves its share; the
    ranks exchange only their statistics, after the run."""
    # more hardware queues than the default 8, so up to 32 resident runs get their own (set
    # before the first CUDA call of the process)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import torch
    from epp import autotune, serve
    from epp.ranks import Ranks, partition
    rk = Ranks.from_env()
    torch.cuda.set_device(rk.local)
    rk.init("nccl")
    if args.mix == "batch":
        specs = serve.batch_mix_requests(args.instances, steps=args.sim_steps)
    else:
        specs = serve.request_stream(args.requests, seed=0, steps=args.sim_steps)
    mine = [specs[i] for i in partition([s_.weight() for s_ in specs], rk.world)[rk.rank]]
    tuner = autotune.Autotuner(device=rk.local, steps=10)
    be = serve.DeviceBackend(device=rk.local, tuner=tuner if args.autotune else None)
    # launch configuration per (dimension, size bucket) of this rank's share, tuned before the clock starts
    tuned = {}
    if args.autotune and not args.native:
        for s_ in mine:
            c = s_.case()
            cp = be.copies(c.n)
            k = autotune.TuneCache.key(tuner.gpu, c.meta["dim"], c.n, False, cp)
            if k not in tuned:
                tuned[k] = tuner.best(c.meta["dim"], c.n, case=c, concurrent=cp)
    # warm-up: one small request of each dimension (module load, first graph build)
    warm = [s for s in serve.request_stream(16, seed=99, n_range=(1e3, 3e3), steps=10)]
    warm = [next(s for s in warm if s.dim == 2), next(s for s in warm if s.dim == 3)]
    for s in warm:
        s.arrival = 0.0
    serve.Server(be).run(serve.make_runs(warm, be))
    runs = serve.make_runs(mine, be)
    rk.barrier()
    clocks = Clocks(rk.local)
    clocks.start()
    if args.native:   # the C-ABI loop (epp_server_*), default launch configuration
        st = serve.serve_native(mine, device=rk.local, budget_bytes=120 * 10**9, co_batch=args.co_batch)
        lat = st.pop("latencies")
    else:
        st = serve.Server(be, budget_bytes=120 * 10**9, co_batch=args.co_batch).run(runs)
        lat = [r.latency for r in runs if r.latency is not None]
    clk = clocks.stop()
    plain_runs = serve.make_runs(mine, be)
    rk.barrier()
    if args.native:
        plain = serve.serve_native(mine, device=rk.local, budget_bytes=120 * 10**9, max_active=1)
        lat_plain = plain.pop("latencies")
    else:
        plain = serve.Server(be, budget_bytes=120 * 10**9, max_active=1).run(plain_runs)
        lat_plain = [r.latency for r in plain_runs if r.latency is not None]
    n_p = [r.case.n for r in runs]
    mine_stats = {"served": st, "plain": plain, "lat": lat, "lat_plain": lat_plain, "particles": n_p,
                  "tuned": {k: list(v) for k, v in tuned.items()}, "clocks": clk}
    every = rk.gather(mine_stats)
    rk.finish()
    if rk.rank != 0:
        return

    def pooled(key, lat_key):
        done = sum(e[key]["completed"] for e in every)
        span = max(e[key]["makespan_s"] for e in every)
        lat = np.array([x for e in every for x in e[lat_key]] or [0.0])
        return {"completed": done, "makespan_s": span, "sims_per_s": done / span if span > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_mean_s": float(lat.mean()),
                "peak_resident_bytes_per_gpu": max(e[key]["peak_resident_bytes"] for e in every),
                "max_concurrent_per_gpu": max(e[key]["max_concurrent"] for e in every)}

    served, plain_all = pooled("served", "lat"), pooled("plain", "lat_plain")
    n_all = [n for e in every for n in e["particles"]]
    h2d = sum(n * 4 * 18 for n in n_all)
    if args.mix == "batch":
        workload = ("the batched form's %d-instance 2D mix as requests arriving at once (width U[0.5,1.5] m, "
                    "height U[1.0,2.5] m, dx=0.01 m)" % len(specs))
    else:
        workload = ("%d requests, Poisson mean 50/s, 70%% 2D / 30%% 3D, fluid log-uniform 1e3-1e6, "
                    "aspect U[0.5,2.5]" % len(specs))
    out = {"metric": "served sims/s (%s, %d steps per simulation)"
                     % ("256-instance mix" if args.mix == "batch" else "Poisson request stream", args.sim_steps),
           "value": served["sims_per_s"], "unit": "sims/s", "n_gpus": rk.world, "steps": args.sim_steps,
           "warmup": 1, "ms_per_step": None, "higher_is_better": True,
           "scaling": "strong" if rk.world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic request stream (numpy default_rng(0)): arrivals, sizes and aspects seeded",
           "config": {"workload": workload, "requests": len(specs), "stream_priorities": "by size",
                      "requests_2d": sum(1 for s in specs if s.dim == 2),
                      "requests_3d": sum(1 for s in specs if s.dim == 3),
                      "particles_total": int(sum(n_all)), "particles_range": [min(n_all), max(n_all)],
                      "hbm_budget_bytes_per_gpu": 120 * 10**9, "chunk_steps": 100,
                      "co_batching": bool(args.co_batch),
                      "loop": "native C ABI (epp_server_*)" if args.native else "Python (epp.serve.Server)",
                      "parallelism": ("requests split over %d GPUs by expected work" % rk.world) if rk.world > 1
                      else "single GPU"},
           "latency_p50_s": served["latency_p50_s"], "latency_p99_s": served["latency_p99_s"],
           "served": served,
           "plain_path": dict(plain_all, method="same trace, one request at a time per GPU (max_active = 1), same kernels"),
           "speedup_vs_plain": served["sims_per_s"] / plain_all["sims_per_s"],
           "p99_vs_plain": served["latency_p99_s"] / plain_all["latency_p99_s"],
           "autotune": {k: {"family": v[0], "block_threads": v[1]} for e in every for k, v in e["tuned"].items()},
           "gpu_launches": 6 * args.sim_steps * len(specs),
           "clocks": every[0]["clocks"],
           "e2e": {"value": served["sims_per_s"], "unit": "sims/s",
                   "h2d_bytes_per_step": int(h2d / args.sim_steps / len(specs)), "d2h_bytes_per_step": 0,
                   "note": "serving is end to end: each request's upload, search, steps and integrals read-back "
                           "are inside the makespan"}}
    print(json.dumps(out))


def main():
    args = parse()
    # more hardware queues than the default 8 for the serve leg's concurrent streams (set before
    # the first CUDA call of the process)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if args.impl == "reference":
        return run_reference(args)
    if args.case == "batch":
        return run_batch(args)
    if args.case == "serve":
        return run_serve(args)
    import torch
    import torch.distributed as dist
    from epp import abi, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    case, label = make_case(args.case, args.physics)
    case.meta["label"] = label
    ps, phys = case.ps, case.physics
    dim = case.meta["dim"]
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    dps = DeviceParticleSystem(ps, ns, device=local)
    ctx = dps.ctx
    if args.lanes:
        ctx.set_tuning(args.lanes)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dps.syncto()
    ctx.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY, phys, 0)
    ctx.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    W = max(args.warmup, 3)
    with torch.cuda.stream(stream):
        ctx.step(W, phys)
    ctx.synchronize()
    clocks = Clocks(local)
    # ---- timed region: K steps, L2 flushed before each, device time by CUDA events ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    p0 = ctx.pairs_total()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            if not args.no_flush:
                flush.fill_(float(k))
            starts[k].record(stream)
            ctx.step(1, phys)
            ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = ctx.synchronize(raise_on_status=False)
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    pairs = ctx.pairs_total() - p0
    if world > 1:
        t = torch.tensor([ms, float(pairs)], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms_max, pairs_all = float(tmax[0]), float(t[1])
    else:
        ms_max, pairs_all = ms, float(pairs)
    value = pairs_all / (ms_max / 1e3)

    # ---- per-kernel device times (instrumented step on the same state, same stream) ----
    with torch.cuda.stream(stream):
        stage = np.zeros(len(STAGES))
        nprof = 5
        for _ in range(nprof):
            if not args.no_flush:
                flush.fill_(1.0)
            stage += np.array(ctx.profile_step(phys))
        stage /= nprof
    # 2D family 0 runs the continuity action inside the search pass (the window search): that
    # kernel carries both stages' bytes and the continuity stage is empty
    b_alg = {k: dict(v) for k, v in B_ALG_STAGE.items()}
    kernel_of = dict(KERNEL_OF_STAGE)
    windows = dim == 2 and args.lanes == 0
    if windows or args.lanes not in (0, 64):   # no continuity kernel: its time is in the search pass
        b_alg["search"][dim] += b_alg["continuity"][dim]
        b_alg["continuity"][dim] = 0.0
        if windows:
            kernel_of["search"] = "k_win_build<CPCont> (window search + lists + continuity + density preview)"
            kernel_of["continuity"] = "(none: the continuity action runs inside the window search)"
    # roofline of the dominant kernel: the longest of the step's kernels
    dom_stage = max(STAGES, key=lambda k: stage[STAGES.index(k)])
    dom_ms = float(stage[STAGES.index(dom_stage)])
    n = case.n
    achieved = b_alg[dom_stage][dim] * n / (dom_ms * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tr_case = {}
    try:   # DRAM bytes of one launch of that kernel from an ncu capture of the same workload
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            # only captures of the kernels this run launches (same kernel, same pair action)
            tr_case = {k: v for k, v in json.load(f).get(args.case, {}).items()
                       if k in kernel_of and kernel_key(v.get("kernel", "")) == kernel_key(kernel_of[k])}
            if tr_case.get(dom_stage):
                traffic = tr_case[dom_stage]["bytes_per_launch"]
    except Exception:
        pass
    fp32_peak = fp32_peak_tflops(stream)

    # ---- end to end through the C ABI with host buffers (pinned) ----
    e2e = run_e2e(dps, case, args.steps, stream)
    if world > 1:   # whole job: every rank's pairs over the slowest rank's host time
        t = torch.tensor([e2e["value"] * e2e["seconds"], e2e["seconds"]], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(t[:1], op=dist.ReduceOp.SUM)
        dist.all_reduce(tmax[1:], op=dist.ReduceOp.MAX)
        e2e["value"] = float(t[0]) / float(tmax[1])
        e2e["seconds"] = float(tmax[1])
        e2e["note"] += "; pairs summed over %d ranks, time of the slowest" % world

    integ = ctx.integrals(phys)
    dps.close()
    del flush
    torch.cuda.empty_cache()
    if rank == 0:
        step_bytes = B_ALG_STEP[dim] * n
        step_ms = ms_max / args.steps
        out = {
            "metric": "SPH pair-interactions/s",
            "value": value,
            "unit": "pair-interactions/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": W,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (dam-break lattice generated in-process, hydrostatic density)",
            "config": plain_config(case, label, world, not args.no_flush),
            "pairs_per_step": pairs_all / args.steps / world,
            "step_hbm_gbs_algorithmic": step_bytes / (step_ms * 1e-3) / 1e9,
            "step_roofline_frac": step_bytes / (step_ms * 1e-3) / 1e9 / peak,
            # per fused step: momentum+integrate+bin, scan, scatter, rank+gather, search, continuity
            # (2D family 0 and the other families run the continuity action inside the search pass)
            "gpu_launches": (6 if (args.lanes == 0 and dim == 3) or args.lanes == 64 else 5) * args.steps
                            + (2 * (args.steps // phys.filter_interval) if phys.filter_interval else 0),
            "roofline": {"bound": "hbm", "kernel": kernel_of[dom_stage], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                         else "fallback 6650 GB/s (of fallback)",
                         "algorithmic_bytes_per_particle": b_alg[dom_stage][dim],
                         "kernel_ms": round(dom_ms, 5),
                         "stage_ms": dict(zip(STAGES, [round(x, 5) for x in stage])),
                         "stage_frac": {k: round(b_alg[k][dim] * n / (stage[STAGES.index(k)] * 1e-3) / 1e9
                                                 / peak, 4) for k in STAGES if b_alg[k][dim] > 0},
                         "frac_of_nominal_8tbs": achieved / 8000.0,
                         "limiter": "instruction issue and neighbour-gather latency, not DRAM bandwidth (ncu: "
                                    "DRAM 4-18% busy in the pair kernels; profiles/)",
                         "compute": compute_roof(tr_case, stage, fp32_peak, clk, kernel_of)},
            "clocks": clk,
            "e2e": e2e,
            "device_status": st,
            "integrals": {k: integ[k] for k in ("mass_total", "kinetic", "potential", "internal", "max_speed")},
        }
        if world == 1:
            try:
                sample = case
                if dim == 3:   # the 3D oracle keeps 100 neighbour columns: sample a smaller block
                    sample = casegen.dam_break_3d(dx=0.01, max_neighbour_number=1)
                    sample.meta["label"] = "3D dam break dx=0.01 (600k fluid), same physics"
                cb = cpu_reference(sample, steps_budget_s=10.0, max_steps=1000)
                out["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as exc:  # reported, not fatal
                out["cpu_baseline"] = {"value": None, "error": str(exc)}
            try:   # 2D: this workload; 3D: the dx = 0.01 block (the FP64 oracle at 6.2M particles is slow)
                dcase = make_case(args.case, args.physics)[0] if dim == 2 else casegen.dam_break_3d(dx=0.01, max_neighbour_number=1)
                out["energy_drift"] = energy_drift_fp64(dcase, 100 if dim == 2 else 10, device=local)
            except Exception as exc:
                out["energy_drift"] = {"error": str(exc)}
            if args.parity:
                try:
                    out["parity"] = parity_block(args, dim, local)
                except Exception as exc:
                    out["parity"] = {"error": repr(exc)}
            if args.served and args.case == "2d" and args.physics == "benchmark":
                try:
                    out["3d"] = measure_3d(local)
                except Exception as exc:
                    out["3d"] = {"error": repr(exc)}
                try:
                    out["batch"] = measure_batch(local, steps=50, warmup=3, instances=256)
                except Exception as exc:
                    out["batch"] = {"error": repr(exc)}
                try:
                    out["serve"] = serve_legs(local, args, out["batch"])
                except Exception as exc:
                    out["serve"] = {"error": repr(exc)}
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def parity_block(args, dim, device):
    """Untimed: the workload's state after 10 fused steps checked against the oracle (cell list,
    neighbour sets, dρ/dt and dv/dt against FP32 and FP64); 3D uses the dx = 0.02 tank."""
    from epp import casegen
    from scale_parity import scale_parity
    t0 = time.perf_counter()
    if dim == 2:
        pcase = casegen.dam_break_2d(dx=0.002 if args.case == "2d" else 0.02, max_neighbour_number=40,
                                     physics=args.physics)
        r = scale_parity(pcase, 40, warm_steps=10, device=device)
    else:
        pcase = casegen.dam_break_3d(dx=0.02, max_neighbour_number=100)
        r = scale_parity(pcase, 100, warm_steps=10, device=device)
    out = {"case": "2D dam break dx=%g" % pcase.meta["dx"] if dim == 2 else "3D dam break dx=0.02 (3.2x1x1 tank)",
           "particles": r["particles"], "scan_tiles": r["scan_tiles"], "cells": r["cells"], "ncount": r["ncount"],
           "sets": r["sets"], "sets_rows_compared": r["sets_rows_compared"],
           "drho_term_vs_fp32": r["drho"]["term_vs_fp32"], "dv_term_vs_fp32": r["dv"]["term_vs_fp32"],
           "drho_rel": r["drho"]["rel_vs_fp32"], "dv_rel": r["dv"]["rel_vs_fp32"],
           "vs_fp64": {"drho_term": r["drho"]["term_vs_fp64"], "dv_term": r["dv"]["term_vs_fp64"],
                       "drho_rel": r["drho"]["rel_vs_fp64"], "dv_rel": r["dv"]["rel_vs_fp64"],
                       "reference_fp32_drho_rel": r["drho"]["oracle_fp32_rel_vs_fp64"],
                       "reference_fp32_dv_rel": r["dv"]["oracle_fp32_rel_vs_fp64"]},
           "floors": {"drho": r["drho"]["floor"], "dv": r["dv"]["floor"]},
           "bar": "bit-exact cells/sets; term-scale error < 1e-5",
           "warm_steps": r["warm_steps"], "seconds": time.perf_counter() - t0}
    out["within_bar"] = bool(r["cells"] and r["sets"] and r["drho"]["term_vs_fp32"] < 1e-5
                             and r["dv"]["term_vs_fp32"] < 1e-5)
    return out


def plain_instance_ms(cases, device, stream, k=20):
    """Device ms per step of each case alone on the plain path: one context sized for the largest
    case, every case uploaded, searched, stepped 3 times untimed and `k` times timed (epp_step
    graph, CUDA events on the context's stream)."""
    import torch
    from epp import abi, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem
    big = max(cases, key=lambda c: c.n)
    ns1 = NeighbourSystem(big.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    plain = DeviceParticleSystem(big.ps, ns1, device=device)
    pctx = plain.ctx
    pctx.set_stream(stream.cuda_stream)
    per_step = []
    for c in cases:
        q = c.ps
        pctx.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, plain.cmap)
        pctx.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY, c.physics, 0)
        with torch.cuda.stream(stream):
            pctx.step(3, c.physics)
        torch.cuda.synchronize()
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a_.record(stream)
            pctx.step(k, c.physics)
            b_.record(stream)
        torch.cuda.synchronize()
        per_step.append(a_.elapsed_time(b_) / k)
    plain.close()
    return per_step


def measure_3d(device, steps=20, warmup=3):
    """3D leg of the 2D line: the 3D dam break at dx = 0.005 m (4.8M fluid particles, 3-layer
    walls: 6.2M), the plain path, `steps` timed steps with the L2 flushed before each."""
    import torch
    from epp import abi, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem
    t_leg = time.perf_counter()
    case = casegen.dam_break_3d(dx=0.005, max_neighbour_number=1)
    phys = case.physics
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    dps = DeviceParticleSystem(case.ps, ns, device=device)
    ctx = dps.ctx
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dps.syncto()
    ctx.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY, phys, 0)
    with torch.cuda.stream(stream):
        ctx.step(warmup, phys)
    ctx.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    p0 = ctx.pairs_total()
    clocks = Clocks(device)
    torch.cuda.synchronize()
    clocks.start()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            ctx.step(1, phys)
            ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = ctx.synchronize(raise_on_status=False)
    ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
    pairs = ctx.pairs_total() - p0
    with torch.cuda.stream(stream):
        stage = np.mean([ctx.profile_step(phys) for _ in range(3)], axis=0)
    dps.close()
    del flush
    torch.cuda.empty_cache()
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    step_ms = ms / steps
    gbs = B_ALG_STEP[3] * case.n / (step_ms * 1e-3) / 1e9
    return {"metric": "SPH pair-interactions/s", "value": pairs / (ms * 1e-3), "unit": "pair-interactions/s",
            "steps": steps, "warmup": warmup, "ms_per_step": step_ms,
            "config": {"workload": "3D dam break dx=0.005 (4.8M fluid)", "particles": case.n,
                       "fluid": case.meta["n_fluid"], "walls": case.meta["n_wall"], "cells": case.meta["n_cells"],
                       "resort": "every step", "l2": "flushed (256 MB write) before every timed step"},
            "pairs_per_step": pairs / steps,
            "step_hbm_gbs_algorithmic": gbs, "step_roofline_frac": gbs / peak,
            "stage_ms": dict(zip(STAGES, [round(float(x), 5) for x in stage])),
            "gpu_launches": 6 * steps, "clocks": clk, "device_status": st,
            "leg_seconds": time.perf_counter() - t_leg}


def measure_batch(device, steps=50, warmup=3, instances=256, sim_steps=2000):
    """Batch leg of the 2D line: the seeded mix of `instances` uneven 2D dam breaks (width
    U[0.5, 1.5] m, height U[1.0, 2.5] m, dx = 0.01 m, each with its own c0 and dt) stepped as one
    batch, every pass one launch over all instances; sims/s at `sim_steps` steps per simulation
    from `steps` timed steps (L2 flushed before each), against the plain path running the same
    instances one at a time (device time per instance step, 20 steps each)."""
    import torch
    from epp import abi, autotune, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem
    import oracle_lib
    from helpers import config_for
    SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
    t_leg = time.perf_counter()
    b = casegen.dam_break_batch(instances, seed=0, dx=0.01)
    phys = b.physics
    ns = NeighbourSystem(b.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    tuned, tune_ms = autotune.tune_case(b, n_instances=b.n_instances, inst=(b.inst_dt, b.inst_c0), steps=5,
                                        device=device)
    dps = DeviceParticleSystem(b.ps, ns, device=device, n_instances=b.n_instances)
    ctx = dps.ctx
    ctx.set_instance_physics(b.inst_dt, b.inst_c0)
    ctx.set_block_threads(tuned[1])
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dps.syncto()
    ctx.search(SYM, CONT, phys, 0)
    e0 = [energy(x) for x in ctx.instance_integrals(phys, b.n_instances)]
    with torch.cuda.stream(stream):
        ctx.step(warmup, phys)
    ctx.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    clocks = Clocks(device)
    torch.cuda.synchronize()
    clocks.start()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            ctx.step(1, phys)
            ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = ctx.synchronize(raise_on_status=False)
    ms = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
    e1 = [energy(x) for x in ctx.instance_integrals(phys, b.n_instances)]
    dps.close()
    del flush
    step_ms = ms / steps
    sims_s = b.n_instances / (sim_steps * step_ms * 1e-3)
    cases = [casegen.dam_break_2d(dx=0.01, column=col, max_neighbour_number=1) for col in b.meta["columns"]]
    per_step = plain_instance_ms(cases, device, stream)
    plain_sims_s = len(cases) / (sim_steps * sum(per_step) * 1e-3)
    # energy drift against the FP64 oracle: the smallest and the largest instance, same steps
    S = warmup + steps
    order = sorted(range(len(cases)), key=lambda k: cases[k].n)
    drift = {}
    oracle_lib.set_threads(os.cpu_count() or 1)
    for k in (order[0], order[-1]):
        c = casegen.dam_break_2d(dx=0.01, column=b.meta["columns"][k], max_neighbour_number=60)
        nso = NeighbourSystem(c.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=60)
        o = oracle_lib.Oracle(config_for(c.ps, nso, max_cell_particles=64), 64)
        q = c.ps
        o.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, q.column_map())
        o.search(SYM, CONT, c.physics)
        o0 = energy(o.integrals(c.physics))
        o.step(S, c.physics)
        o1 = energy(o.integrals(c.physics))
        dg, do = (e1[k] - e0[k]) / abs(e0[k]), (o1 - o0) / abs(o0)
        drift[str(k)] = {"particles": c.n, "gpu_fp32": dg, "oracle_fp64": do, "abs_diff": abs(dg - do)}
    return {"metric": "batched sims/s (%d-instance 2D dam-break mix, %d steps per simulation)"
                      % (b.n_instances, sim_steps),
            "value": sims_s, "unit": "sims/s", "steps": steps, "warmup": warmup, "ms_per_step": step_ms,
            "config": {"workload": "%d uneven 2D dam breaks, width U[0.5,1.5] m, height U[1.0,2.5] m, dx=0.01 m, "
                                   "seed 0" % b.n_instances, "particles": b.n,
                       "fluid_per_instance": [min(b.meta["inst_n_fluid"]), max(b.meta["inst_n_fluid"])],
                       "cells": b.meta["n_cells"], "dt": "per instance (0.1 h / c0_k)",
                       "l2": "flushed (256 MB write) before every timed step"},
            "plain_path": {"sims_per_s": plain_sims_s, "ms_per_instance_step_mean": float(np.mean(per_step)),
                           "ms_per_instance_step": [round(x, 5) for x in per_step],
                           "method": "each instance alone on the plain path (epp_step graph), 20 steps timed by "
                                     "CUDA events per instance, summed over the instances"},
            "speedup_vs_plain": sims_s / plain_sims_s,
            "autotune": {"family": tuned[0], "block_threads": tuned[1], "resort_every": 1},
            "energy_drift": {"steps": S, "bar": 1e-4, "instances": drift,
                             "max_abs_diff": max(v["abs_diff"] for v in drift.values())},
            "gpu_launches": 5 * steps, "clocks": clk, "device_status": st,
            "leg_seconds": time.perf_counter() - t_leg}


def serve_legs(device, args, batch):
    """Serve leg of the 2D line.  (a) The batch leg's instance mix as requests arriving at once,
    co-batched by the Python serving loop (2000 steps each): sims/s and p50/p99 completion latency;
    its one-at-a-time baseline is the batch leg's per-instance plain-path device time, run in FIFO
    order (completion of request k = sum of the first k runs; host work not counted, which favours
    the baseline).  (b) The first `args.leg_requests` requests of the seeded Poisson stream (mean
    50 req/s, 70% 2D / 30% 3D, 1e3-1e6 fluid particles, 2000 steps each) served with continuous
    batching under a 120 GB budget and, for the baseline, the same requests one at a time
    (max_active = 1); default launch configuration (no autotuner), both measured on the host clock."""
    from epp import serve
    t_leg = time.perf_counter()
    be = serve.DeviceBackend(device=device)
    out = {}
    # warm-up: one small request of each dimension (module load, first graph builds)
    warm = [s for s in serve.request_stream(16, seed=99, n_range=(1e3, 3e3), steps=10)]
    warm = [next(s for s in warm if s.dim == 2), next(s for s in warm if s.dim == 3)]
    for s in warm:
        s.arrival = 0.0
    serve.Server(be).run(serve.make_runs(warm, be))
    # (a) the instance mix, co-batched
    specs = serve.batch_mix_requests(256, steps=2000)
    runs = serve.make_runs(specs, be)
    clocks = Clocks(device)
    clocks.start()
    st = serve.Server(be, budget_bytes=120 * 10**9, co_batch=True).run(runs)
    clk = clocks.stop()
    per = batch["plain_path"]["ms_per_instance_step"] if isinstance(batch, dict) and "plain_path" in batch else None
    mix = {"workload": "the batch leg's 256-instance mix as requests arriving at once, 2000 steps each, co-batched",
           "sims_per_s": st["sims_per_s"], "latency_p50_s": st["latency_p50_s"], "latency_p99_s": st["latency_p99_s"],
           "makespan_s": st["makespan_s"], "completed": st["completed"], "clocks": clk}
    if per:
        done = np.cumsum(np.array(per) * 2000 * 1e-3)
        mix["plain_path"] = {"sims_per_s": len(per) / float(done[-1]), "latency_p50_s": float(np.percentile(done, 50)),
                             "latency_p99_s": float(np.percentile(done, 99)),
                             "method": "per-instance plain-path device time x 2000 steps, FIFO one at a time"}
        mix["speedup_vs_plain"] = mix["sims_per_s"] / mix["plain_path"]["sims_per_s"]
    out["mix"] = mix
    # (b) the Poisson stream
    specs = serve.request_stream(32, seed=0, steps=2000)[: args.leg_requests]
    runs = serve.make_runs(specs, be)
    clocks = Clocks(device)
    clocks.start()
    st = serve.Server(be, budget_bytes=120 * 10**9, co_batch=True).run(runs)
    clk = clocks.stop()
    plain_runs = serve.make_runs(specs, be)
    pl = serve.Server(be, budget_bytes=120 * 10**9, max_active=1).run(plain_runs)
    n_p = [r.case.n for r in runs]
    out["stream"] = {"workload": "first %d requests of the seeded Poisson stream (mean 50 req/s, 70%% 2D / 30%% 3D, "
                                 "fluid log-uniform 1e3-1e6, 2000 steps each)" % len(specs),
                     "requests_2d": sum(1 for s in specs if s.dim == 2),
                     "requests_3d": sum(1 for s in specs if s.dim == 3),
                     "particles_range": [min(n_p), max(n_p)],
                     "sims_per_s": st["sims_per_s"], "latency_p50_s": st["latency_p50_s"],
                     "latency_p99_s": st["latency_p99_s"], "makespan_s": st["makespan_s"],
                     "max_concurrent": st["max_concurrent"], "clocks": clk,
                     "plain_path": {"sims_per_s": pl["sims_per_s"], "latency_p50_s": pl["latency_p50_s"],
                                    "latency_p99_s": pl["latency_p99_s"],
                                    "method": "same requests one at a time (max_active = 1), same kernels"},
                     "speedup_vs_plain": st["sims_per_s"] / pl["sims_per_s"] if pl["sims_per_s"] else None}
    out["budget_bytes"] = 120 * 10**9
    out["leg_seconds"] = time.perf_counter() - t_leg
    return out


def fp32_peak_tflops(stream):
    """FP32 (non-tensor) roof measured here: cuBLAS SGEMM 8192^3 with TF32 off, best of 5, CUDA
    events on `stream`."""
    import torch
    prev = torch.get_float32_matmul_precision()
    torch.set_float32_matmul_precision("highest")
    try:
        n = 8192
        with torch.cuda.stream(stream):
            a = torch.randn(n, n, device="cuda")
            b = torch.randn(n, n, device="cuda")
            c = torch.empty(n, n, device="cuda")
            for _ in range(2):
                torch.matmul(a, b, out=c)
            best = float("inf")
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                torch.matmul(a, b, out=c)
                e1.record(stream)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
        del a, b, c
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.set_float32_matmul_precision(prev)


def compute_roof(tr_case, stage, fp32_peak, clk, kernel_of=None):
    """Second roof of the three pair kernels: FP32 flops and warp instructions per launch (ncu
    instruction-mix capture of the same workload) over this run's kernel times, against the
    measured SGEMM FP32 rate and the issue rate 148 SMs x 4 schedulers x the sampled SM clock."""
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    issue_peak = 148 * 4 * mhz * 1e6
    out = {"fp32_peak_tflops": fp32_peak, "fp32_peak_source": "cuBLAS SGEMM 8192^3, TF32 off (of measured)",
           "issue_peak_warp_inst_per_s": issue_peak, "issue_clock_mhz": mhz, "stages": {}}
    for st in B_ALG_STAGE:
        e = tr_case.get(st) or {}
        ms = float(stage[STAGES.index(st)])
        if "flops_per_launch" not in e or ms <= 0:
            continue
        tf = e["flops_per_launch"] / (ms * 1e-3) / 1e12
        out["stages"][st] = {"kernel": (kernel_of or KERNEL_OF_STAGE)[st], "kernel_ms": round(ms, 5),
                             "flops_per_launch": e["flops_per_launch"], "achieved_tflops": tf,
                             "fp32_frac": tf / fp32_peak,
                             "warp_inst_per_launch": e["warp_inst_per_launch"],
                             "issue_frac": e["warp_inst_per_launch"] / (ms * 1e-3) / issue_peak}
    return out


def energy_drift_fp64(case, steps, device=0):
    """Energy check on this workload: relative energy drift (kinetic + potential + internal,
    FP64 integrals) over `steps` fused steps, the FP32 CUDA path against the FP64 oracle from the
    same initial state; the bar is |drift_gpu - drift_fp64| <= 1e-4."""
    from epp import abi, casegen
    from epp.algorithm import DeviceParticleSystem
    from epp.classes import NeighbourSystem
    import oracle_lib
    from helpers import config_for
    SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
    phys = case.physics
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    d = DeviceParticleSystem(case.ps, ns, device=device)
    d.syncto()
    d.ctx.search(SYM, CONT, phys, 0)
    g0 = energy(d.ctx.integrals(phys))
    d.ctx.step(steps, phys)
    g1 = energy(d.ctx.integrals(phys))
    d.close()
    dim = case.meta["dim"]
    nso = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40 if dim == 2 else 100)
    oracle_lib.set_threads(os.cpu_count() or 1)
    o = oracle_lib.Oracle(config_for(case.ps, nso, max_cell_particles=64 if dim == 2 else 128), 64)
    q = case.ps
    o.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, q.column_map())
    o.search(SYM, CONT, phys)
    o0 = energy(o.integrals(phys))
    o.step(steps, phys)
    o1 = energy(o.integrals(phys))
    dg, do = (g1 - g0) / abs(g0), (o1 - o0) / abs(o0)
    return {"steps": steps, "particles": case.n, "gpu_fp32": dg, "oracle_fp64": do, "abs_diff": abs(dg - do),
            "bar": 1e-4, "within_bar": abs(dg - do) <= 1e-4}


def pinned_copy(a, order="F"):
    """A copy of numpy array `a` in page-locked host memory with the given element order; returns
    (torch tensor that owns the memory, numpy view of it)."""
    import torch
    tt = {np.dtype(np.float32): torch.float32, np.dtype(np.int32): torch.int32}[a.dtype]
    t = torch.empty(max(a.size, 1), dtype=tt, pin_memory=True)
    v = t.numpy()[: a.size].reshape(a.shape, order=order)
    v[...] = a
    assert t.is_pinned() and np.shares_memory(v, t.numpy())
    assert v.flags.f_contiguous if order == "F" else v.flags.c_contiguous
    return t, v


def run_e2e(dps, case, K, stream, reps=5):
    """Same metric through the public C ABI with host buffers in page-locked memory (allocated once,
    column-major like the reference's matrices): upload, initial search, K x (epp_step + that
    step's FP64 integrals read back, one step in flight), download.  Host clock; the region is
    repeated `reps` times (each continuing from the last state) and the median is reported, with
    its phases (each phase ends with the device idle).  Pairs: the K steps' searches only."""
    ps = dps.host
    ctx = dps.ctx
    phys = case.physics
    keep = []
    bufs = {}
    for name, arr, order in (("ip", ps.int_properties, "F"), ("fp", ps.float_properties, "F"),
                             ("alive", ps.is_alive, "C"), ("cell", ps.cell_index, "C")):
        t, v = pinned_copy(np.asarray(arr), order)
        keep.append(t)
        bufs[name] = v
    ip, fp, alive, cell = bufs["ip"], bufs["fp"], bufs["alive"], bufs["cell"]
    ctx.download(alive, cell, ip, fp, dps.cmap)   # the host matrices hold the current state
    runs = []
    for _ in range(reps):
        ctx.synchronize()
        t0 = time.perf_counter()
        ctx.upload(ps.n_particles, alive, cell, ip, fp, dps.cmap)
        ctx.synchronize()
        t1 = time.perf_counter()
        ctx.search(1, 1, phys, 0)
        ctx.synchronize()
        t2 = time.perf_counter()
        p0 = ctx.pairs_total()
        t2b = time.perf_counter()
        pending = None
        for _ in range(K):
            ctx.step(1, phys)
            t = ctx.integrals_async(phys)
            if pending is not None:
                ctx.integrals_wait(pending)
            pending = t
        ctx.integrals_wait(pending)
        t3 = time.perf_counter()
        p1 = ctx.pairs_total()
        t3b = time.perf_counter()
        ctx.download(alive, cell, ip, fp, dps.cmap)
        t4 = time.perf_counter()
        total = (t4 - t0) - (t2b - t2) - (t3b - t3)   # the pair-count reads are bookkeeping
        runs.append({"seconds": total, "pairs": p1 - p0, "upload_s": t1 - t0, "search_s": t2 - t1,
                     "steps_with_readback_s": t3 - t2b, "download_s": t4 - t3b})
    runs.sort(key=lambda r: r["seconds"])
    med = runs[len(runs) // 2]
    cm = dps.cmap
    d = case.meta["dim"]
    ncols_f = sum(w for c, w in [(cm.position, d), (cm.velocity, d), (cm.dvelocity, d), (cm.mass, 1), (cm.volume, 1),
                                 (cm.density, 1), (cm.ddensity, 1), (cm.pressure, 1), (cm.h, 1), (cm.gap, 1)]
                  if c >= 0)
    ncols_i = 2 + sum(1 for c in (cm.tag, cm.is_movable, cm.n_count, cm.instance) if c >= 0)
    n = ps.n_particles
    h2d = n * 4 * (ncols_f + ncols_i)
    d2h = n * 4 * (ncols_f + ncols_i - (1 if cm.instance >= 0 else 0)) + 72 * K
    return {"value": med["pairs"] / med["seconds"], "unit": "pair-interactions/s",
            "h2d_bytes_per_step": int(h2d / K), "d2h_bytes_per_step": int(d2h / K), "seconds": med["seconds"],
            "steps": K, "repeats": reps, "phases_s": {k: med[k] for k in ("upload_s", "search_s",
                                                                          "steps_with_readback_s", "download_s")},
            "seconds_all": [round(r["seconds"], 6) for r in runs],
            "host_buffers": "page-locked, column-major, allocated once",
            "note": "upload + initial search + K x (step + integrals read back, one step in flight) + download, "
                    "host clock, median of %d; pairs of the K steps' searches" % reps}


if __name__ == "__main__":
    main()
