"""CFL time step (epp_physics.cfl > 0): every step's dt = cfl h_min / (c0 + max|v|) of the state it
starts from, reduced on the device inside the step (FP64 from the FP32 velocities, rounded once).

The reference steps with a fixed dt (example/collapse_dry/same/main.jl:68); the CFL rule is the
time step the benchmark's 3D and batched cases name.  Bars:

* max|v|, the FP64 CFL dt of a state and the FP32 dt the next step takes equal the oracle's for
  the same state, bit for bit (max and min do not depend on the summation order);
* a free-running CFL trajectory stays with the oracle's (positions to 1e-6 of the domain,
  simulated time and next dt to 1e-5 relative: the FP32 velocities differ by rounding);
* in a batch every instance takes its own CFL dt with its own c0, and ends bit-identical to the
  same case run alone.
"""
import numpy as np
import pytest

from epp import abi, casegen
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem
from helpers import config_for
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
CFL = 0.2


def cfl_physics(phys, cfl=CFL):
    p = abi.epp_physics.from_buffer_copy(phys)
    p.cfl = cfl
    return p


def stirred_case(dx=0.04, seed=3):
    """The 2D dam break with a seeded velocity field in the fluid (up to 4 m/s), so that max|v|
    moves the CFL dt well away from the fixed one."""
    case = casegen.dam_break_2d(dx=dx, max_neighbour_number=40)
    rng = np.random.default_rng(seed)
    v = case.ps["VelocityVec"]
    fl = case.ps["Tag"] == casegen.FLUID_TAG
    v[fl] = rng.uniform(-2.0, 2.0, (int(fl.sum()), 2)).astype(np.float32)
    case.ps["VelocityVec"] = v
    return case


def device_and_oracle(case, precision=32):
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40)
    d = DeviceParticleSystem(case.ps, ns)
    d.syncto()
    o = Oracle(config_for(case.ps, ns, max_cell_particles=64), precision)
    ps = case.ps
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, ps.column_map())
    return d, o


def test_cfl_dt_and_max_speed_equal_the_oracle():
    case = stirred_case()
    phys = cfl_physics(case.physics)
    d, _ = device_and_oracle(case)
    d.ctx.search(SYM, CONT, phys, 0)
    d.ctx.step(5, phys)
    gi = d.ctx.integrals(phys)
    g_dt, g_t = d.ctx.step_dt(phys)
    d.asyncto()
    # the oracle loaded with the device's state
    o = Oracle(d.config, 32)
    ps = d.host
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, d.cmap)
    o.search(SYM, CONT, phys)
    oi = o.integrals(phys)
    o_dt, _ = o.step_dt(phys)
    assert gi["max_speed"] == oi["max_speed"] and gi["max_speed"] > 1.0
    assert gi["cfl_dt"] == oi["cfl_dt"]
    assert float(g_dt[0]) == float(np.float32(o_dt))
    assert float(g_dt[0]) == float(np.float32(gi["cfl_dt"]))
    # the dt is the CFL one, not the fixed one
    assert abs(float(g_dt[0]) - case.physics.dt) > 0.02 * case.physics.dt
    assert g_t[0] > 0.0
    d.close()


def test_cfl_trajectory_follows_the_oracle():
    steps = 40
    case = stirred_case()
    phys = cfl_physics(case.physics)
    d, o = device_and_oracle(case)
    d.ctx.search(SYM, CONT, phys, 0)
    o.search(SYM, CONT, phys)
    dt0, _ = d.ctx.step_dt(phys)
    odt0, _ = o.step_dt(phys)
    assert float(dt0[0]) == float(np.float32(odt0))   # same initial state: same first dt
    d.ctx.step(steps, phys)
    o.step(steps, phys)
    g_dt, g_t = d.ctx.step_dt(phys)
    o_dt, o_t = o.step_dt(phys)
    d.asyncto()
    n = case.n
    gx = d.host["PositionVec"].astype(np.float64)
    ox = np.stack([o.field(0, a, n) for a in range(2)], 1)
    assert np.max(np.abs(gx - ox)) < 1e-6
    assert abs(g_t[0] - o_t) <= 1e-5 * o_t
    assert abs(float(g_dt[0]) - o_dt) <= 1e-5 * o_dt
    # the time step really varied along the run
    assert abs(g_t[0] - steps * float(dt0[0])) > 1e-4 * g_t[0]
    # against the FP64 oracle: same trajectory to FP32 rounding
    o64 = Oracle(d.config, 64)
    c2 = stirred_case()
    q = c2.ps
    o64.upload(q.n_particles, q.is_alive, q.cell_index, q.int_properties, q.float_properties, q.column_map())
    o64.search(SYM, CONT, phys)
    o64.step(steps, phys)
    _, t64 = o64.step_dt(phys)
    assert abs(g_t[0] - t64) <= 1e-5 * t64
    d.close()


def test_fixed_dt_time_is_steps_times_dt():
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    d = DeviceParticleSystem(case.ps, ns)
    d.syncto()
    d.ctx.search(SYM, CONT, case.physics, 0)
    d.ctx.step(7, case.physics)
    dt, t = d.ctx.step_dt(case.physics)
    assert float(dt[0]) == case.physics.dt
    assert t[0] == 7 * float(np.float64(np.float32(case.physics.dt)))
    d.close()


def test_cfl_batch_instances_take_their_own_dt_and_equal_alone():
    columns = [(0.5, 1.0), (1.3, 2.4), (0.8, 1.7)]
    dx, steps = 0.04, 25
    b = casegen.dam_break_batch(columns=columns, dx=dx)
    phys = cfl_physics(b.physics)
    ns = NeighbourSystem(b.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    db = DeviceParticleSystem(b.ps, ns, n_instances=b.n_instances)
    db.ctx.set_instance_physics(b.inst_dt, b.inst_c0)
    db.syncto()
    db.ctx.search(SYM, CONT, phys, 0)
    db.ctx.step(steps, phys)
    bdt, bt = db.ctx.step_dt(phys, b.n_instances)
    db.asyncto()
    assert len(set(float(x) for x in bdt)) == len(columns)   # every instance its own dt
    for k, col in enumerate(columns):
        c = casegen.dam_break_2d(dx=dx, column=col, max_neighbour_number=1)
        cphys = cfl_physics(c.physics)
        nsa = NeighbourSystem(c.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        da = DeviceParticleSystem(c.ps, nsa)
        da.syncto()
        da.ctx.search(SYM, CONT, cphys, 0)
        da.ctx.step(steps, cphys)
        adt, at = da.ctx.step_dt(cphys)
        da.asyncto()
        r0, r1 = b.rows[k]
        for name in ("PositionVec", "VelocityVec", "Density", "dDensity"):
            assert np.array_equal(db.host[name][r0:r1], da.host[name]), (k, name)
        assert float(bdt[k]) == float(adt[0]), k
        assert bt[k] == at[0], k
        da.close()
    db.close()


def test_cfl_requires_family_0_and_a_valid_number():
    from epp.lib import EppError
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    d = DeviceParticleSystem(case.ps, ns)
    d.syncto()
    d.ctx.search(SYM, CONT, case.physics, 0)
    bad = cfl_physics(case.physics, -1.0)
    with pytest.raises(EppError) as e:
        d.ctx.step(1, bad)
    assert e.value.code == abi.EPP_ERR_INVALID_ARGUMENT
    d.ctx.set_tuning(4)
    with pytest.raises(EppError) as e:
        d.ctx.step(1, cfl_physics(case.physics))
    assert e.value.code == abi.EPP_ERR_UNSUPPORTED_ACTION
    d.close()
