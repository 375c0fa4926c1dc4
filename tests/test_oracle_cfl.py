"""The oracle's CFL time step (CPU): dt = cfl h_min / (c0 + max|v|) of the state a step starts from,
over the alive fluid particles, in FP64 and rounded once to the system's precision."""
import numpy as np

from epp import abi, casegen
from epp.classes import NeighbourSystem
from helpers import config_for
from oracle_lib import Oracle

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY


def _oracle(case, precision=32):
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40)
    o = Oracle(config_for(case.ps, ns, max_cell_particles=64), precision)
    ps = case.ps
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, ps.column_map())
    o.search(SYM, CONT, case.physics)
    return o


def _cfl(phys, cfl):
    p = abi.epp_physics.from_buffer_copy(phys)
    p.cfl = cfl
    return p


def _expected(case, cfl):
    ps = case.ps
    fl = ps["Tag"] == casegen.FLUID_TAG
    v = ps["VelocityVec"][fl].astype(np.float64)
    vmax = np.sqrt(np.max(np.sum(v * v, axis=1)))
    hmin = float(np.min(ps["H"][fl].astype(np.float64)))
    return np.float32(float(np.float32(cfl)) * hmin / (float(np.float32(case.physics.c0)) + vmax))


def test_cfl_dt_at_rest_is_the_fixed_dt():
    case = casegen.dam_break_2d(dx=0.05, max_neighbour_number=40)
    o = _oracle(case)
    dt, t = o.step_dt(_cfl(case.physics, 0.1))
    assert t == 0.0
    assert np.float32(dt) == _expected(case, 0.1)
    # the reference's dt = 0.1 h / c0 (main.jl:68), to one FP32 ulp (0.1 is not exact in FP32)
    assert abs(dt - case.physics.dt) <= np.spacing(np.float32(case.physics.dt))
    dt_fixed, _ = o.step_dt(case.physics)
    assert np.float32(dt_fixed) == np.float32(case.physics.dt)


def test_cfl_dt_of_a_moving_state_and_the_time_it_adds_up():
    case = casegen.dam_break_2d(dx=0.05, max_neighbour_number=40)
    rng = np.random.default_rng(1)
    v = case.ps["VelocityVec"]
    fl = case.ps["Tag"] == casegen.FLUID_TAG
    v[fl] = rng.uniform(-3.0, 3.0, (int(fl.sum()), 2)).astype(np.float32)
    case.ps["VelocityVec"] = v
    phys = _cfl(case.physics, 0.25)
    o = _oracle(case)
    dt, _ = o.step_dt(phys)
    assert np.float32(dt) == _expected(case, 0.25)
    ig = o.integrals(phys)
    assert np.float32(ig["cfl_dt"]) == np.float32(dt)
    total = 0.0
    for _ in range(6):
        d, _ = o.step_dt(phys)
        total += d
        o.step(1, phys)
    _, t = o.step_dt(phys)
    assert t == total
    # FP64 oracle: the same rule, unrounded
    o64 = _oracle(case, 64)
    d64, _ = o64.step_dt(phys)
    assert abs(d64 - dt) <= 1e-7 * dt
