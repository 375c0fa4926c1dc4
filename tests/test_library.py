"""SPH library options on the CUDA path against the oracle: the four smoothing kernels, the linear
EOS, classic viscosity, sAccelerateMove! and the kernel filter -- the physics of the reference's
own example (example/collapse_dry/same/main.jl:53-144).

Same bars as tests/test_gpu_parity.py: neighbour sets bit-exact; per stage, from identical state,
1e-5 relative to the sum of |terms|; free-running trajectories together to FP32 rounding.
"""
import copy

import numpy as np
import pytest

from epp import abi, casegen
from epp.lib import EppError
from oracle_lib import ORC_FIELD_ACCEL_ABS, ORC_FIELD_DDENSITY_ABS, ORC_FIELD_DENSITY
from test_gpu_parity import REL, cond_err, gpu_fields, make_case, oracle_fields, pair, rel_err, sync_oracle

pytestmark = pytest.mark.gpu

SYM = abi.EPP_CRITERION_SYMMETRY
CONT = abi.EPP_ACTION_DAMBREAK_CONTINUITY
KERNELS = [abi.EPP_KERNEL_WENDLAND_C2, abi.EPP_KERNEL_CUBIC_SPLINE, abi.EPP_KERNEL_GAUSSIAN,
           abi.EPP_KERNEL_WENDLAND_C4]


def with_physics(case, **kw):
    p = copy.copy(case.physics)
    for k, v in kw.items():
        setattr(p, k, v)
    case.physics = p
    return case


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("dim,dx", [(2, 0.04), (3, 0.02)])
def test_kernel_lists_and_continuity(dim, dx, kernel):
    """search! with the kernel cache (iValueGradient!, SPH/Library/Kernel.jl:114-128): the emitted
    nW, nDW, nHInv and dρ/dt against the oracle for each kernel."""
    max_nb = 40 if dim == 2 else 100
    case = with_physics(make_case(dim, dx, max_nb), kernel=kernel)
    dps, o = pair(case, max_nb)
    n = case.n
    dps.ctx.search(SYM, CONT, case.physics, abi.EPP_SEARCH_EMIT_LIST)
    o.search(SYM, CONT, case.physics)
    dps.ctx.synchronize()
    g = gpu_fields(dps)
    r = oracle_fields(o, n, dim)
    assert cond_err(g["drho"], r["drho"], o.field(ORC_FIELD_DDENSITY_ABS, 0, n)) < REL
    ops = make_case(dim, dx, max_nb).ps
    o.download(ops.is_alive, ops.cell_index, ops.int_properties, ops.float_properties, dps.cmap)
    cnt = dps.host["nCount"]
    assert np.array_equal(cnt, ops["nCount"])
    mask = np.arange(max_nb)[None, :] < cnt[:, None]
    # each particle's entries ordered by neighbour id (the sets are equal; compare the values)
    big = np.iinfo(np.int32).max
    oa = np.argsort(np.where(mask, dps.host["nIndex"], big), axis=1, kind="stable")
    ob = np.argsort(np.where(mask, ops["nIndex"], big), axis=1, kind="stable")
    assert np.array_equal(np.take_along_axis(dps.host["nIndex"], oa, 1)[mask],
                          np.take_along_axis(ops["nIndex"], ob, 1)[mask])
    for name in ("nW", "nDW", "nHInv"):
        a = np.take_along_axis(dps.host[name], oa, 1)[mask]
        b = np.take_along_axis(ops[name], ob, 1)[mask]
        assert np.max(np.abs(a - b)) <= 2e-6 * max(np.max(np.abs(b)), 1e-30), name


@pytest.mark.parametrize("dim,dx,options", [
    (2, 0.04, "example"),
    (3, 0.02, dict(kernel=abi.EPP_KERNEL_WENDLAND_C4, eos=abi.EPP_EOS_LINEAR, viscosity=abi.EPP_VISCOSITY_CLASSIC,
                   mu=1e-3, motion=abi.EPP_MOTION_ACCELERATE_MOVE)),
    (2, 0.04, dict(kernel=abi.EPP_KERNEL_GAUSSIAN)),
])
def test_library_stage_parity(dim, dx, options):
    """The example's loop body call by call (main.jl:166-183), each stage from the device state
    loaded into the oracle: density update with the chosen EOS, momentum with the chosen kernel
    and viscosity, the chosen time integration, search + continuity, and the kernel filter."""
    max_nb = 40 if dim == 2 else 100
    if options == "example":
        case = casegen.dam_break_2d(dx=dx, max_neighbour_number=max_nb, physics="example")
    else:
        case = with_physics(make_case(dim, dx, max_nb), **options)
    phys = case.physics
    dps, o = pair(case, max_nb)
    n = case.n
    c = dps.ctx
    c.search(SYM, CONT, phys, 0)
    o.search(SYM, CONT, phys)
    fluid = case.ps["Tag"] == casegen.FLUID_TAG
    for _ in range(2):
        sync_oracle(dps, o, case)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_DENSITY, phys)
        o.selfaction(abi.EPP_ACTION_DAMBREAK_DENSITY, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert np.array_equal(g["rho"], r["rho"].astype(np.float32))
        assert rel_err(g["p"], r["p"], 1.0) < REL
        sync_oracle(dps, o, case)
        c.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
        o.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        dv_abs = np.stack([o.field(ORC_FIELD_ACCEL_ABS, a, n) for a in range(dim)], 1)
        assert cond_err(g["dv"], r["dv"], dv_abs) < REL
        sync_oracle(dps, o, case)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_INTEGRATE, phys)
        o.selfaction(abi.EPP_ACTION_DAMBREAK_INTEGRATE, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert rel_err(g["v"], r["v"], 1e-3) < REL
        assert rel_err(g["x"], r["x"], 1.0) < 1e-6
        sync_oracle(dps, o, case)
        c.search(SYM, CONT, phys, 0)
        o.search(SYM, CONT, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert cond_err(g["drho"], r["drho"], o.field(ORC_FIELD_DDENSITY_ABS, 0, n)) < REL
        sync_oracle(dps, o, case)
        c.interaction(abi.EPP_ACTION_KERNEL_FILTER, phys)
        c.selfaction(abi.EPP_ACTION_KERNEL_FILTER_SELF, phys)
        o.interaction(abi.EPP_ACTION_KERNEL_FILTER, phys)
        o.selfaction(abi.EPP_ACTION_KERNEL_FILTER_SELF, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert rel_err(g["rho"][fluid], r["rho"][fluid], 1.0) < REL
        assert rel_err(g["vol"], r["vol"], 1e-12) < REL
        if phys.eos == abi.EPP_EOS_LINEAR:   # p = c0^2 (rho - rho0) + p0 of the device's own density
            c02 = np.float32(phys.c0) * np.float32(phys.c0)
            expect = c02 * (g["rho"] - np.float32(phys.rho0)) + np.float32(phys.p0)
            assert np.array_equal(g["p"][fluid], expect[fluid])


def test_example_fused_steps_with_filter():
    """epp_step with the example's physics, filter every 20 steps, against the oracle's loop for
    25 steps from the same initial state (the filter runs after step 20 in both), and the filter
    really runs: without it the density differs."""
    dim, dx, steps = 2, 0.04, 25
    case = casegen.dam_break_2d(dx=dx, max_neighbour_number=40, physics="example")
    phys = case.physics
    dps, o = pair(case, 40)
    n = case.n
    dps.ctx.search(SYM, CONT, phys, 0)
    o.search(SYM, CONT, phys)
    dps.ctx.step(steps, phys)
    o.step(steps, phys)
    dps.ctx.synchronize()
    g, r = gpu_fields(dps), oracle_fields(o, n, dim)
    assert np.max(np.abs(g["x"] - r["x"])) < 1e-6
    assert np.max(np.abs(g["rho"] - r["rho"]) / r["rho"]) < 1e-5
    assert np.max(np.abs(g["v"] - r["v"])) <= 1e-3 * max(np.max(np.abs(r["v"])), 1e-3)
    gi, oi = dps.ctx.integrals(phys), o.integrals(phys)
    e_g = gi["kinetic"] + gi["potential"] + gi["internal"]
    e_o = oi["kinetic"] + oi["potential"] + oi["internal"]
    assert abs(e_g - e_o) <= 1e-5 * abs(e_o)
    # same run without the filter: the densities differ
    nof = casegen.dam_break_2d(dx=dx, max_neighbour_number=40, physics="example")
    p2 = copy.copy(phys)
    p2.filter_interval = 0
    d2, _ = pair(nof, 40)
    d2.ctx.search(SYM, CONT, p2, 0)
    d2.ctx.step(steps, p2)
    d2.ctx.synchronize()
    assert not np.array_equal(gpu_fields(d2)["rho"], g["rho"])


def test_filter_pending_and_family_errors():
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=40, physics="example")
    phys = case.physics
    dps, _ = pair(case, 40)
    c = dps.ctx
    c.search(SYM, CONT, phys, 0)
    c.interaction(abi.EPP_ACTION_KERNEL_FILTER, phys)
    with pytest.raises(EppError) as e:
        c.search(SYM, CONT, phys, 0)
    assert e.value.code == abi.EPP_ERR_STATE
    c.selfaction(abi.EPP_ACTION_KERNEL_FILTER_SELF, phys)
    c.search(SYM, CONT, phys, 0)
    c.set_tuning(4)
    with pytest.raises(EppError) as e:
        c.step(1, phys)
    assert e.value.code == abi.EPP_ERR_UNSUPPORTED_ACTION
    bad = copy.copy(phys)
    bad.kernel = 9
    c.set_tuning(0)
    with pytest.raises(EppError) as e:
        c.step(1, bad)
    assert e.value.code == abi.EPP_ERR_INVALID_ARGUMENT


DW, BAL, CLS = abi.EPP_PRESSURE_DENSITY_WEIGHTED, abi.EPP_PRESSURE_BALANCED, abi.EPP_PRESSURE_CLASSIC
EXTRAP = abi.EPP_WALL_PRESSURE_EXTRAPOLATE
PRESSURE_OPTIONS = [
    (2, 0.04, dict(pressure_ff=DW, pressure_fw=DW, tensile=1)),
    (3, 0.02, dict(pressure_ff=BAL, pressure_fw=CLS, tensile=1, kernel=abi.EPP_KERNEL_WENDLAND_C4)),
    (2, 0.04, dict(kernel=abi.EPP_KERNEL_CUBIC_SPLINE, wall_pressure=EXTRAP)),
    (3, 0.02, dict(pressure_ff=DW, wall_pressure=EXTRAP)),
]


@pytest.mark.parametrize("dim,dx,options", PRESSURE_OPTIONS)
def test_pressure_stage_parity(dim, dx, options):
    """Pressure.jl on the CUDA path, each stage from the device state loaded into the oracle: the
    wall-pressure extrapolation (iExtrapolatePressure! + sExtrapolatePressure!), then momentum with
    the chosen pressure terms and iPressureCorrection, integration and search + continuity."""
    max_nb = 40 if dim == 2 else 100
    case = with_physics(make_case(dim, dx, max_nb), **options)
    phys = case.physics
    dps, o = pair(case, max_nb)
    n = case.n
    c = dps.ctx
    c.search(SYM, CONT, phys, 0)
    o.search(SYM, CONT, phys)
    wall = case.ps["Tag"][:n] == casegen.WALL_TAG
    for _ in range(2):
        sync_oracle(dps, o, case)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_DENSITY, phys)
        o.selfaction(abi.EPP_ACTION_DAMBREAK_DENSITY, phys)
        if options.get("wall_pressure") == EXTRAP:
            sync_oracle(dps, o, case)
            c.interaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE, phys)
            c.selfaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, phys)
            o.interaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE, phys)
            o.selfaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, phys)
            c.synchronize()
            g, r = gpu_fields(dps), oracle_fields(o, n, dim)
            # a weighted mean of non-negative terms: relative error of a few FP32 roundings
            assert rel_err(g["p"][wall], r["p"][wall], 1.0) < REL
            assert np.array_equal(g["p"][~wall], r["p"][~wall].astype(np.float32))
        sync_oracle(dps, o, case)
        c.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
        o.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        dv_abs = np.stack([o.field(ORC_FIELD_ACCEL_ABS, a, n) for a in range(dim)], 1)
        assert cond_err(g["dv"], r["dv"], dv_abs) < REL
        sync_oracle(dps, o, case)
        c.selfaction(abi.EPP_ACTION_DAMBREAK_INTEGRATE, phys)
        o.selfaction(abi.EPP_ACTION_DAMBREAK_INTEGRATE, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert rel_err(g["x"], r["x"], 1.0) < 1e-6
        sync_oracle(dps, o, case)
        c.search(SYM, CONT, phys, 0)
        o.search(SYM, CONT, phys)
        c.synchronize()
        g, r = gpu_fields(dps), oracle_fields(o, n, dim)
        assert cond_err(g["drho"], r["drho"], o.field(ORC_FIELD_DDENSITY_ABS, 0, n)) < REL


@pytest.mark.parametrize("dim,dx,options", PRESSURE_OPTIONS)
def test_pressure_fused_steps(dim, dx, options):
    """epp_step with the pressure options (the extrapolation inside the fused step, after each
    density preview) against the oracle's loop from the same initial state."""
    max_nb = 40 if dim == 2 else 100
    steps = 20
    case = with_physics(make_case(dim, dx, max_nb), **options)
    phys = case.physics
    dps, o = pair(case, max_nb)
    n = case.n
    dps.ctx.search(SYM, CONT, phys, 0)
    o.search(SYM, CONT, phys)
    dps.ctx.step(steps, phys)
    o.step(steps, phys)
    dps.ctx.synchronize()
    g, r = gpu_fields(dps), oracle_fields(o, n, dim)
    assert np.max(np.abs(g["x"] - r["x"])) < 1e-6
    assert np.max(np.abs(g["rho"] - r["rho"]) / r["rho"]) < 1e-5
    assert np.max(np.abs(g["v"] - r["v"])) <= 1e-3 * max(np.max(np.abs(r["v"])), 1e-3)
    assert np.max(np.abs(g["p"] - r["p"])) <= 1e-4 * max(np.max(np.abs(r["p"])), 1.0)
    if options.get("wall_pressure") == EXTRAP:   # the walls' pressure is not the EOS of their density
        wall = case.ps["Tag"][:n] == casegen.WALL_TAG
        eos = copy.copy(phys)
        eos.wall_pressure = abi.EPP_WALL_PRESSURE_EOS
        d2, _ = pair(with_physics(make_case(dim, dx, max_nb), **dict(options, wall_pressure=0)), max_nb)
        d2.ctx.search(SYM, CONT, eos, 0)
        d2.ctx.step(steps, eos)
        d2.ctx.synchronize()
        assert not np.array_equal(gpu_fields(d2)["p"][wall], g["p"][wall])


def test_pressure_option_errors():
    case = with_physics(make_case(2, 0.04, 40), wall_pressure=EXTRAP)
    phys = case.physics
    dps, _ = pair(case, 40)
    c = dps.ctx
    c.search(SYM, CONT, phys, 0)
    c.interaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE, phys)
    with pytest.raises(EppError) as e:   # the sums are indexed by the current order
        c.search(SYM, CONT, phys, 0)
    assert e.value.code == abi.EPP_ERR_STATE
    with pytest.raises(EppError) as e:
        c.step(1, phys)
    assert e.value.code == abi.EPP_ERR_STATE
    c.selfaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, phys)
    c.search(SYM, CONT, phys, 0)
    for fam in (1, 4):
        c.set_tuning(fam)
        with pytest.raises(EppError) as e:
            c.step(1, phys)
        assert e.value.code == abi.EPP_ERR_UNSUPPORTED_ACTION
    c.set_tuning(0)
    for field, value in (("pressure_ff", 4), ("pressure_fw", -1), ("tensile", 2), ("wall_pressure", 2)):
        bad = copy.copy(phys)
        setattr(bad, field, value)
        with pytest.raises(EppError) as e:
            c.step(1, bad)
        assert e.value.code == abi.EPP_ERR_INVALID_ARGUMENT, field
    # the tensile correction reads the Gap column: refused when the upload did not map it
    dps.cmap.gap = -1
    dps.syncto()
    c.search(SYM, CONT, case.physics, 0)
    t = copy.copy(phys)
    t.tensile = 1
    with pytest.raises(EppError) as e:
        c.step(1, t)
    assert e.value.code == abi.EPP_ERR_INVALID_ARGUMENT
