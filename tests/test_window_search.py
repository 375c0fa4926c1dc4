"""The 2D window search (the default family-0 search pass in 2D) against the tiled list build
(EPP_TUNING_LISTS).

Both build the same neighbour lists in the same order (stencil rows, then cell order, then id order
inside a cell): the window search tests each particle's own stencil-row windows from cell rows
staged in shared memory and runs the continuity action while it writes the list, the tiled build
tests whole tiles and leaves continuity to a list pass.  Neighbour counts and stored lists are
identical and every sum agrees to FP32 rounding (the compiler may contract a multiply and an add
into one fused operation differently in the two kernels).  Checked after fused steps and per-call
actions, on multi-tile grids, warps that cross cell-row ends and particles with more neighbours than
a list keeps (read from their stencil)."""
import numpy as np
import pytest

from epp import abi, casegen
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem

pytestmark = pytest.mark.gpu

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
FIELDS = ("PositionVec", "VelocityVec", "Density", "dDensity", "Pressure", "Volume", "nCount", "dVelocityVec")


def pair_of_contexts(case):
    """(window search, tiled list build) contexts of the same case."""
    out = []
    for tuning in (0, abi.EPP_TUNING_LISTS):
        ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        d = DeviceParticleSystem(case.ps, ns)
        d.ctx.set_tuning(tuning)
        d.syncto()
        out.append(d)
    return out


def host_fields(d):
    d.asyncto()
    return {k: d.host[k].copy() for k in FIELDS}


FLOORS = {"PositionVec": 1.0, "VelocityVec": 1e-2, "Density": 1.0, "dDensity": 1.0, "Pressure": 1.0,
          "Volume": 1e-9, "dVelocityVec": 1.0}


def assert_same(a, b, what):
    """nCount exactly; the rest to FP32 rounding: |a - b| <= 1e-5 max(|b|, floor)."""
    assert np.array_equal(a["nCount"], b["nCount"]), (what, "nCount")
    for k in FIELDS:
        if k == "nCount":
            continue
        x, y = a[k].astype(np.float64), b[k].astype(np.float64)
        assert np.all(np.isfinite(x)) and np.all(np.isfinite(y)), (what, k)
        err = np.max(np.abs(x - y) / np.maximum(np.abs(y), FLOORS[k])) if x.size else 0.0
        assert err <= 1e-5, (what, k, err, int(np.sum(x != y)))


def case_of(dx, h_factor):
    return casegen.dam_break_2d(dx=dx, h_factor=h_factor, max_neighbour_number=1)


@pytest.mark.parametrize("dx,h_factor,steps", [(0.04, 1.5, 20), (0.02, 1.5, 10), (0.005, 1.5, 3),
                                               (0.04, 3.0, 4), (0.02, 2.2, 3)])
def test_fused_steps_match(dx, h_factor, steps):
    case = case_of(dx, h_factor)
    phys = case.physics
    m, l = pair_of_contexts(case)
    for d in (m, l):
        d.ctx.search(SYM, CONT, phys, 0)
        d.ctx.step(steps, phys)
        d.ctx.synchronize()
    a, b = host_fields(m), host_fields(l)
    assert_same(a, b, "fused steps")
    n = case.n
    ca, ia = m.ctx.neighbour_lists(n, 64)
    cb, ib = l.ctx.neighbour_lists(n, 64)
    assert np.array_equal(ca, cb)
    stored = (ca > 0) & (ca <= 64)
    if h_factor >= 3:   # more neighbours than a list keeps: read from the stencil, not stored
        assert stored.sum() < n and np.all(ia[ca > 64] == 0) and np.all(ib[cb > 64] == 0)
    assert np.all(ia[stored, 0] != 0)
    assert np.array_equal(ia[stored], ib[stored])
    for d in (m, l):
        d.close()


@pytest.mark.parametrize("h_factor", [1.5, 3.0])
def test_per_call_actions_match(h_factor):
    """search! (count only and continuity), interaction! (momentum, neighbour count, kernel filter,
    pressure extrapolation) and selfaction! on both forms."""
    case = case_of(0.04, h_factor)
    phys = case.physics
    m, l = pair_of_contexts(case)
    for d in (m, l):
        c = d.ctx
        c.search(SYM, abi.EPP_ACTION_NONE, phys, 0)
        c.interaction(abi.EPP_ACTION_COUNT_NEIGHBOURS, phys)
        c.selfaction(abi.EPP_ACTION_ZERO_DVELOCITY)
        c.search(SYM, CONT, phys, 0)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_DENSITY, phys)
        c.interaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE, phys)
        c.selfaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, phys)
        c.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_INTEGRATE, phys)
        c.search(SYM, CONT, phys, 0)
        c.interaction(abi.EPP_ACTION_KERNEL_FILTER, phys)
        c.selfaction(abi.EPP_ACTION_KERNEL_FILTER_SELF, phys)
        c.synchronize()
    assert_same(host_fields(m), host_fields(l), "per-call actions")
    for d in (m, l):
        d.close()


def test_default_criterion_and_example_physics_match():
    """The default criterion (dr^2 <= gap^2) and the example's physics (CubicSpline, classic
    viscosity, kernel filter every 20 steps inside epp_step)."""
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1, physics="example")
    phys = case.physics
    m, l = pair_of_contexts(case)
    for d in (m, l):
        d.ctx.search(abi.EPP_CRITERION_DEFAULT, abi.EPP_ACTION_NONE, phys, 0)
        d.ctx.interaction(abi.EPP_ACTION_COUNT_NEIGHBOURS, phys)
        d.ctx.search(SYM, CONT, phys, 0)
        d.ctx.step(25, phys)
        d.ctx.synchronize()
    assert_same(host_fields(m), host_fields(l), "example physics")
    for d in (m, l):
        d.close()
