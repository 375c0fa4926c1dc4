"""The oracle's restatements of src/SPH/Library/Pressure.jl against a direct numpy evaluation of
the reference's formulas on the oracle's own neighbour lists and kernel cache, in FP64:
iClassicPressure!, iBalancedPressure!, iDensityWeightedPressure! (:24-83), iPressureCorrection
(:10-22), iExtrapolatePressure! (:85-131) and sExtrapolatePressure! (:133-150).

The reference's own test of these functions (test/SPH/LibraryTest.jl:86-113) calls each of them
on a 9-particle system without checking values, so there is no golden vector to pin them; this
test checks the oracle's C++ against a second, independent statement of the same formulas.
"""
import copy

import numpy as np
import pytest

from epp import abi, casegen
from epp.classes import NeighbourSystem
from helpers import config_for
from oracle_lib import ORC_FIELD_DVELOCITY, ORC_FIELD_PRESSURE, Oracle, kernel

FLUID, WALL = casegen.FLUID_TAG, casegen.WALL_TAG
SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY


def _oracle(case, phys):
    ps = case.ps
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40)
    o = Oracle(config_for(ps, ns), 64)
    cmap = ps.column_map()
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, cmap)
    o.search(SYM, CONT, phys)
    o.download(ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, cmap)
    return o, ps


def _lists(ps):
    n = ps.n_particles
    cnt = ps["nCount"]
    nb = ps["nIndex"] - 1   # 1-based in the reference layout
    nb_max = nb.shape[1]
    rvec = ps["nRVec"].reshape(n, nb_max, -1) if ps["nRVec"].ndim == 2 else ps["nRVec"]
    return cnt, nb, ps["nR"], ps["nW"], ps["nDW"], ps["nHInv"], rvec


def _pressure(form, p, rho, i, j):
    if form == abi.EPP_PRESSURE_CLASSIC:
        return p[i] / (rho[i] * rho[i]) + p[j] / (rho[j] * rho[j])
    if form == abi.EPP_PRESSURE_BALANCED:
        return (p[i] + p[j]) / (rho[i] * rho[j])
    return 2 * (p[i] * rho[i] + p[j] * rho[j]) / ((rho[i] + rho[j]) * rho[i] * rho[j])


@pytest.mark.parametrize("pff,pfw,tensile,kind", [
    (abi.EPP_PRESSURE_DEFAULT, abi.EPP_PRESSURE_DEFAULT, 0, abi.EPP_KERNEL_WENDLAND_C2),
    (abi.EPP_PRESSURE_DENSITY_WEIGHTED, abi.EPP_PRESSURE_DENSITY_WEIGHTED, 1, abi.EPP_KERNEL_WENDLAND_C2),
    (abi.EPP_PRESSURE_BALANCED, abi.EPP_PRESSURE_CLASSIC, 1, abi.EPP_KERNEL_CUBIC_SPLINE),
])
def test_pressure_forms(pff, pfw, tensile, kind):
    case = casegen.dam_break_2d(dx=0.05, max_neighbour_number=40)
    phys = copy.copy(case.physics)
    phys.alpha = phys.beta = 0.0   # artificial viscosity off: dv is the pressure term alone
    phys.pressure_ff, phys.pressure_fw, phys.tensile, phys.kernel = pff, pfw, tensile, kind
    ps = case.ps
    # a non-uniform pressure field so that every form differs
    ps["Pressure"] = (ps["Pressure"] + 50.0 * np.sin(7.0 * ps["PositionVec"][:, 0])).astype(np.float32)
    o, ps = _oracle(case, phys)
    o.interaction(abi.EPP_ACTION_DAMBREAK_MOMENTUM, phys)
    n = ps.n_particles
    got = np.stack([o.field(ORC_FIELD_DVELOCITY, a, n) for a in range(2)], 1)
    cnt, nb, r, w, dw, hinv, rvec = _lists(ps)
    tag, m = ps["Tag"], ps["Mass"].astype(np.float64)
    p, rho, gap = (ps[k].astype(np.float64) for k in ("Pressure", "Density", "Gap"))
    ff_form = abi.EPP_PRESSURE_CLASSIC if pff == abi.EPP_PRESSURE_DEFAULT else pff
    fw_form = abi.EPP_PRESSURE_BALANCED if pfw == abi.EPP_PRESSURE_DEFAULT else pfw
    expect = np.zeros((n, 2))
    for i in range(n):
        if tag[i] != FLUID:
            continue
        for k in range(cnt[i]):
            j = nb[i, k]
            if tag[j] not in (FLUID, WALL):
                continue
            t = _pressure(ff_form if tag[j] == FLUID else fw_form, p, rho, i, j)
            if tensile:
                t += abs(t) * 0.01 * w[i, k] / kernel(kind, 2, 0.5 * (gap[i] + gap[j]), hinv[i, k])[0]
            t *= -m[j] * dw[i, k] / r[i, k]
            expect[i] += t * rvec[i, k]
    scale = np.max(np.abs(expect))
    assert scale > 0   # the lists read back here are FP32 copies of the oracle's FP64 values
    assert np.max(np.abs(got - expect)) <= 1e-6 * scale


def test_extrapolate_pressure():
    case = casegen.dam_break_2d(dx=0.05, max_neighbour_number=40)
    phys = copy.copy(case.physics)
    o, ps = _oracle(case, phys)
    o.interaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE, phys)
    o.selfaction(abi.EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF, phys)
    n = ps.n_particles
    got = o.field(ORC_FIELD_PRESSURE, 0, n)
    cnt, nb, r, w, dw, hinv, rvec = _lists(ps)
    tag = ps["Tag"]
    p, rho, vol = (ps[k].astype(np.float64) for k in ("Pressure", "Density", "Volume"))
    g = np.array(phys.gravity[:2], np.float64)
    p0 = float(phys.p0)
    expect = p.copy()
    walls_with_fluid = 0
    for i in range(n):
        if tag[i] != WALL:
            continue
        wv = wvp = 0.0
        for k in range(cnt[i]):
            j = nb[i, k]
            if tag[j] != FLUID:
                continue
            g_dot_x = float(rvec[i, k] @ g)
            a = w[i, k] * vol[j]
            wv += a
            wvp += a * (max(p[j], p0) + max(rho[j] * g_dot_x, p0))
        expect[i] = wvp / wv if wv > 0 else p0
        walls_with_fluid += wv > 0
    assert walls_with_fluid > 0
    wall = tag[:n] == WALL
    # the lists and state read back here are FP32 copies of the oracle's FP64 values
    assert np.max(np.abs(got[wall] - expect[wall])) <= 1e-6 * max(np.max(np.abs(expect[wall])), 1.0)
    assert np.array_equal(got[~wall], p[~wall])   # fluid pressure untouched
