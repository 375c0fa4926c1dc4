"""Parity of the CUDA path against the oracle at full problem sizes (test infrastructure).

One state of a dam break is produced on the device (an initial search and `warm_steps` fused
steps, so velocities and density rates are not zero), then checked against the oracle loaded
with that same state:

* cell list: counts, exclusive offsets and the particles of every cell sorted by id, bit-exact;
* neighbour sets: the lists the search pass built (what every pair pass of a step reads),
  against the nIndex/nCount columns of the oracle's search, bit-exact as sets;
* dρ/dt of the step's search (continuity) and dv/dt of the next step's momentum pass, each
  stage recomputed by the FP32 oracle (the reference's arithmetic and neighbour order) and by
  the FP64 oracle from the device's input to that stage.

Two error measures are reported for the physics:
* `term`: |a - b| / (sum of |terms| of the particle's sum) -- the rounding scale of an FP32 sum,
  the bar (1e-5) the parity tests assert against the FP32 oracle;
* `rel`: |a - b| / max(|b|, floor), plain relative error with a stated floor (g for dv/dt,
  1e-6 rho0 c0 / h for dρ/dt), as max and 99.9th percentile.
Against FP64 the same measures are given for the device and for the FP32 oracle, so the device's
error can be read against the reference's own FP32 error.

The oracle's neighbour lists are the reference's: it keeps `max_nb` columns per particle.
"""
import copy

import numpy as np

from epp import abi, casegen
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem
from oracle_lib import (ORC_FIELD_ACCEL, ORC_FIELD_ACCEL_ABS, ORC_FIELD_DDENSITY, ORC_FIELD_DDENSITY_ABS,
                        ORC_FIELD_NCOUNT, Oracle)

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY


def term_err(a, b, scale, floor=1e-30):
    a, b, scale = (np.asarray(v, np.float64) for v in (a, b, scale))
    return float(np.max(np.abs(a - b) / np.maximum(scale, floor))) if a.size else 0.0


def rel_stats(a, b, floor):
    """max and 99.9th percentile of |a - b| / max(|b|, floor)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if not a.size:
        return {"max": 0.0, "p999": 0.0}
    e = (np.abs(a - b) / np.maximum(np.abs(b), floor)).ravel()
    return {"max": float(e.max()), "p999": float(np.quantile(e, 0.999))}


def neighbour_pairs(counts, ids):
    """Sorted (row, neighbour id) pairs of per-row neighbour lists: counts[n], ids[n, k]."""
    counts = np.asarray(counts)
    k = ids.shape[1]
    keep = np.arange(k)[None, :] < np.minimum(counts, k)[:, None]
    rows = np.broadcast_to(np.arange(len(counts))[:, None], ids.shape)[keep].astype(np.int64)
    nb = ids[keep].astype(np.int64)
    key = rows * (1 << 32) + nb
    key.sort()
    return key


class ScaleParity:
    """Device system and FP32 / FP64 oracles for one case."""

    def __init__(self, case, max_nb, device=0, max_cell_particles=None):
        self.case = case
        self.dim = case.meta["dim"]
        self.n = case.n
        self.max_nb = max_nb
        ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=max_nb)
        self.dps = DeviceParticleSystem(case.ps, ns, device=device)
        self.dps.physics = case.physics
        cfg = type(self.dps.config).from_buffer_copy(self.dps.config)
        cfg.max_cell_particles = max_cell_particles or (64 if self.dim == 2 else 128)
        self.cfg = cfg
        self.o32 = Oracle(cfg, 32)
        self.o64 = Oracle(cfg, 64)

    def close(self):
        self.dps.close()

    def _load(self, o, drho=None):
        """The device's current state into oracle `o`, searched (cells, lists, kernel cache);
        dDensity set to `drho` (None: zero before the search, so the search's continuity action
        leaves this state's dρ/dt)."""
        ps = self.dps.host
        o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, self.dps.cmap)
        if drho is None:
            o.set_field(ORC_FIELD_DDENSITY, np.zeros(ps.n_particles))
        o.search(SYM, CONT, self.case.physics)
        if drho is not None:
            o.set_field(ORC_FIELD_DDENSITY, drho)

    def run(self, warm_steps=10):
        c, phys, n, dim = self.dps.ctx, self.case.physics, self.n, self.dim
        self.dps.syncto()
        c.search(SYM, CONT, phys, 0)
        if warm_steps:
            c.step(warm_steps, phys)
        c.synchronize()
        out = {"particles": n, "cells_total": int(self.case.meta["n_cells"]), "warm_steps": warm_steps}
        # ---- cell list and neighbour sets at this state ----
        self.dps.asyncto()
        ps = self.dps.host
        alive = ps.is_alive[:n].copy()
        gc, go, gi = c.cell_stats()
        g_cnt, g_ids = c.neighbour_lists(n, self.max_nb)
        g_drho = ps["dDensity"].astype(np.float64).copy()
        self._load(self.o32)
        oc, oo, oi = self.o32.cell_stats(int(alive.sum()))
        out["scan_tiles"] = int((len(gc) + 1 + 2047) // 2048)
        out["cells"] = bool(np.array_equal(gc, oc) and np.array_equal(go, oo) and np.array_equal(gi, oi))
        o_cnt = self.o32.field(ORC_FIELD_NCOUNT, 0, n).astype(np.int32)
        ops = self._oracle_host()
        self.o32.download(ops.is_alive, ops.cell_index, ops.int_properties, ops.float_properties, self.dps.cmap)
        bi = ops.basic_index
        o_ids = ops.int_properties[:n, bi["nIndex"] - 1: bi["nIndex"] - 1 + self.max_nb]
        # rows whose neighbours the device stores (the others read their stencil in every pass)
        full = ((g_ids[:, 0] != 0) | (g_cnt == 0)) & (g_cnt <= self.max_nb) & (o_cnt <= self.max_nb)
        out["ncount"] = bool(np.array_equal(g_cnt, o_cnt))
        out["sets"] = bool(out["ncount"] and np.array_equal(
            neighbour_pairs(np.where(full, g_cnt, 0), g_ids), neighbour_pairs(np.where(full, o_cnt, 0), o_ids)))
        out["sets_rows_compared"] = int(full.sum())
        out["pairs"] = int(g_cnt.sum())
        # ---- dρ/dt of this state's search (continuity), FP32 and FP64 oracle ----
        fluid = (ps["Tag"][:n] == casegen.FLUID_TAG) & (alive == 1)
        r32 = self.o32.field(ORC_FIELD_DDENSITY, 0, n)
        s32 = self.o32.field(ORC_FIELD_DDENSITY_ABS, 0, n)
        self._load(self.o64)
        r64 = self.o64.field(ORC_FIELD_DDENSITY, 0, n)
        s64 = self.o64.field(ORC_FIELD_DDENSITY_ABS, 0, n)
        h = float(self.case.meta["h"])
        floor_drho = 1e-6 * phys.rho0 * phys.c0 / h
        m = alive == 1
        out["drho"] = {
            "term_vs_fp32": term_err(g_drho[m], r32[m], s32[m]),
            "rel_vs_fp32": rel_stats(g_drho[m], r32[m], floor_drho),
            "term_vs_fp64": term_err(g_drho[m], r64[m], s64[m]),
            "rel_vs_fp64": rel_stats(g_drho[m], r64[m], floor_drho),
            "oracle_fp32_term_vs_fp64": term_err(r32[m], r64[m], s64[m]),
            "oracle_fp32_rel_vs_fp64": rel_stats(r32[m], r64[m], floor_drho),
            "floor": floor_drho,
        }
        # ---- dv/dt of the next step's momentum pass from this state ----
        c.set_accel_output(True)
        self._load(self.o32, g_drho)
        self._load(self.o64, g_drho)
        c.step(1, phys)
        self.o32.step(1, phys)
        self.o64.step(1, phys)
        c.synchronize()
        acc = c.accel(n, dim)
        c.set_accel_output(False)
        a32 = np.stack([self.o32.field(ORC_FIELD_ACCEL, a, n) for a in range(dim)], 1)
        a64 = np.stack([self.o64.field(ORC_FIELD_ACCEL, a, n) for a in range(dim)], 1)
        s32 = np.stack([self.o32.field(ORC_FIELD_ACCEL_ABS, a, n) for a in range(dim)], 1)
        s64 = np.stack([self.o64.field(ORC_FIELD_ACCEL_ABS, a, n) for a in range(dim)], 1)
        g = max(abs(float(x)) for x in phys.gravity) or 9.81
        f = fluid
        out["dv"] = {
            "term_vs_fp32": term_err(acc[f], a32[f], s32[f]),
            "rel_vs_fp32": rel_stats(acc[f], a32[f], g),
            "term_vs_fp64": term_err(acc[f], a64[f], s64[f]),
            "rel_vs_fp64": rel_stats(acc[f], a64[f], g),
            "oracle_fp32_term_vs_fp64": term_err(a32[f], a64[f], s64[f]),
            "oracle_fp32_rel_vs_fp64": rel_stats(a32[f], a64[f], g),
            "floor": g,
        }
        return out

    def _oracle_host(self):
        """A host particle system of the case's layout for the oracle's download."""
        return copy.deepcopy(self.dps.host)


def scale_parity(case, max_nb, warm_steps=10, device=0, max_cell_particles=None):
    sp = ScaleParity(case, max_nb, device=device, max_cell_particles=max_cell_particles)
    try:
        return sp.run(warm_steps)
    finally:
        sp.close()
