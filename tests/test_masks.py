"""2D stencil-row masks (the default family-0 pair passes in 2D) against the neighbour-list passes.

Both forms visit every particle's neighbours in the same order (stencil rows, then cell order,
then id order inside a cell), so every sum is the same: the state after fused steps, per-call
actions and the neighbour sets must be bit-identical between a context on masks and one set to
EPP_TUNING_LISTS, including multi-tile grids, warps that cross cell-row ends and particles whose
stencil rows hold more than 32 candidates (read from their stencil)."""
import numpy as np
import pytest

from epp import abi, casegen
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem

pytestmark = pytest.mark.gpu

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
FIELDS = ("PositionVec", "VelocityVec", "Density", "dDensity", "Pressure", "Volume", "nCount", "dVelocityVec")


def pair_of_contexts(case):
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


def assert_same(a, b, what):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), (what, k)


@pytest.mark.parametrize("dx,h_factor,steps", [(0.04, 1.5, 20), (0.02, 1.5, 10), (0.04, 3.0, 4)])
def test_fused_steps_bit_identical(dx, h_factor, steps):
    case = casegen.dam_break_2d(dx=dx, h_factor=h_factor, max_neighbour_number=1)
    phys = case.physics
    m, l = pair_of_contexts(case)
    for d in (m, l):
        d.ctx.search(SYM, CONT, phys, 0)
        d.ctx.step(steps, phys)
        d.ctx.synchronize()
    a, b = host_fields(m), host_fields(l)
    assert_same(a, b, "fused steps")
    n = case.n
    ca, ia = m.ctx.neighbour_lists(n, 160)
    cb, ib = l.ctx.neighbour_lists(n, 160)
    assert np.array_equal(ca, cb)
    stored = ia[:, 0] != 0
    if h_factor > 2:   # stencil rows of more than 32 candidates: read from the stencil, not stored
        assert stored.sum() < n
    keep = stored & (ib[:, 0] != 0)
    assert np.array_equal(ia[keep], ib[keep])
    for d in (m, l):
        d.close()


def test_per_call_actions_bit_identical():
    """search! (count only and continuity), interaction! (momentum, neighbour count, kernel filter,
    pressure extrapolation) and selfaction! on both forms."""
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
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


def test_default_criterion_and_example_physics_bit_identical():
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
