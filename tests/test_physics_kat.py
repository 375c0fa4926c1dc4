"""Physics known answers, on the oracle (CPU) and on the CUDA path (GPU).

The reference's own library test (test/SPH/LibraryTest.jl:10-114) calls the physics functions
without assertions, so these answers come from the physics itself, independent of any
restatement of the reference's code:

* hydrostatic column: in the interior of the initial dam-break column (hydrostatic density on the
  Tait EOS, at rest) the pressure gradient balances gravity: |dv/dt| < 1% of g (the consistency
  error of the SPH gradient at h = 1.5 dx is about 0.5-0.8%);
* momentum: classic pressure and artificial viscosity act in equal and opposite pairs
  (Pressure.jl:24-41, Viscosity.jl:28-52): with no gravity and no walls, sum m_i dv_i/dt = 0 and
  for two particles m_i a_i = -m_j a_j, to FP32 rounding of the terms;
* continuity (Continuity.jl:23-47): under a uniform translation every v_i - v_j vanishes, so
  dρ/dt = 0 exactly;
* kernels (src/SPH/Kernel/*.jl): dW/dr equals the central difference of W for all four kernels in
  2D and 3D, and the CUDA path's dW/dr (read through a two-particle continuity rate) equals it.
"""
import numpy as np
import pytest

from epp import abi, casegen
from epp.classes import Domain2D, Domain3D, NeighbourSystem, ParticleSystem
from helpers import config_for
from oracle_lib import ORC_FIELD_DDENSITY, ORC_FIELD_DVELOCITY, Oracle, kernel

SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY
MOM = abi.EPP_ACTION_DAMBREAK_MOMENTUM
KERNELS = [abi.EPP_KERNEL_WENDLAND_C2, abi.EPP_KERNEL_CUBIC_SPLINE, abi.EPP_KERNEL_GAUSSIAN,
           abi.EPP_KERNEL_WENDLAND_C4]


def tiny_case(pos, vel, rho, h, physics, tag=None, pad=0.5):
    """A particle system of the given particles (fluid unless `tag` says otherwise) in a domain
    around them; mass = rho V with V = h^dim / 1.5^dim."""
    pos = np.asarray(pos, np.float32)
    n, dim = pos.shape
    lo, hi = pos.min(0) - pad, pos.max(0) + pad
    gap = 2.0 * h
    domain = Domain2D(gap, lo[0], lo[1], hi[0], hi[1]) if dim == 2 else \
        Domain3D(gap, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2])
    ints, floats = casegen._layout(dim, 40)
    ps = ParticleSystem(domain, n, ints, floats, {"rho0": 1000.0})
    vol = np.full(n, (h / 1.5) ** dim, np.float32)
    rho = np.asarray(rho, np.float32)
    ps["PositionVec"] = pos
    ps["VelocityVec"] = np.asarray(vel, np.float32)
    ps["Density"] = rho
    ps["Volume"] = vol
    ps["Mass"] = (rho * vol).astype(np.float32)
    ps["H"] = np.full(n, h, np.float32)
    ps["Gap"] = np.full(n, h / 1.5, np.float32)
    ps["Tag"] = np.asarray(tag if tag is not None else np.full(n, casegen.FLUID_TAG), np.int32)
    ps["IsMovable"] = (ps["Tag"] == casegen.FLUID_TAG).astype(np.int32)
    B = casegen.tait_b(1000.0, physics.c0, physics.gamma)
    ps["Pressure"] = (B * ((rho.astype(np.float64) / 1000.0) ** physics.gamma - 1.0)).astype(np.float32)
    return casegen.DamBreakCase(ps, domain, physics, {"dim": dim, "h": h, "n_cells": domain.get_n()})


def no_gravity_physics(dim, h, kernel_kind=abi.EPP_KERNEL_WENDLAND_C2):
    c0 = 30.0
    g = (0.0, 0.0, 0.0)
    return abi.make_physics(float(np.float32(0.1 * h / c0)), c0=c0, gravity=g, kernel=kernel_kind)


def oracle_of(case, precision=32):
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40)
    o = Oracle(config_for(case.ps, ns, max_cell_particles=64), precision)
    ps = case.ps
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, ps.column_map())
    return o


def device_of(case):
    from epp.algorithm import DeviceParticleSystem
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=40)
    d = DeviceParticleSystem(case.ps, ns)
    d.syncto()
    return d


def dv_of(case, on_gpu):
    """dVelocity of one interaction!(momentum) after search!(continuity) (no gravity added)."""
    n, dim = case.n, case.meta["dim"]
    if not on_gpu:
        o = oracle_of(case)
        o.search(SYM, CONT, case.physics)
        o.interaction(MOM, case.physics)
        return np.stack([o.field(ORC_FIELD_DVELOCITY, a, n) for a in range(dim)], 1)
    d = device_of(case)
    d.ctx.search(SYM, CONT, case.physics, 0)
    d.ctx.selfaction(abi.EPP_ACTION_ZERO_DVELOCITY)
    d.ctx.interaction(MOM, case.physics)
    d.ctx.synchronize()
    d.asyncto()
    out = d.host["dVelocityVec"].astype(np.float64).copy()
    d.close()
    return out


def drho_of(case, on_gpu):
    """dDensity of search!(continuity) from zero."""
    n = case.n
    case.ps["dDensity"] = np.zeros(n, np.float32)
    if not on_gpu:
        o = oracle_of(case)
        o.search(SYM, CONT, case.physics)
        return o.field(ORC_FIELD_DDENSITY, 0, n)
    d = device_of(case)
    d.ctx.search(SYM, CONT, case.physics, 0)
    d.ctx.synchronize()
    d.asyncto()
    out = d.host["dDensity"].astype(np.float64).copy()
    d.close()
    return out


def hydrostatic_interior(on_gpu):
    case = casegen.dam_break_2d(dx=0.02, max_neighbour_number=40)
    du = dv_of(case, on_gpu)
    g = np.array(case.physics.gravity[:2], np.float64)
    acc = du + g
    x, h = case.ps["PositionVec"], case.meta["h"]
    W, H = case.meta["column"]
    fl = case.ps["Tag"] == casegen.FLUID_TAG
    inner = fl & (x[:, 0] > 3 * h) & (x[:, 0] < W - 3 * h) & (x[:, 1] > 3 * h) & (x[:, 1] < H - 3 * h)
    assert inner.sum() > 3000
    return np.max(np.linalg.norm(acc[inner], axis=1)) / np.linalg.norm(g)


def momentum_balance(on_gpu, dim):
    rng = np.random.default_rng(5 + dim)
    h = 0.03
    n = 60 if dim == 2 else 120
    pos = rng.uniform(0.0, 3.0 * h * (4 if dim == 2 else 2), (n, dim))
    vel = rng.normal(0.0, 0.5, (n, dim))
    rho = 1000.0 * (1.0 + rng.uniform(-0.01, 0.01, n))
    case = tiny_case(pos, vel, rho, h, no_gravity_physics(dim, h))
    du = dv_of(case, on_gpu)
    m = case.ps["Mass"].astype(np.float64)[:, None]
    total = np.abs((m * du).sum(0)).max()
    scale = np.abs(m * du).sum(0).max()
    return total, scale


def two_particles(on_gpu, dim):
    h = 0.03
    pos = np.zeros((2, dim))
    pos[1, 0] = 0.8 * h
    pos[1, 1] = 0.5 * h
    vel = np.zeros((2, dim))
    vel[0, 0] = 1.0     # approaching: the artificial viscosity acts too
    case = tiny_case(pos, vel, [1003.0, 998.0], h, no_gravity_physics(dim, h))
    du = dv_of(case, on_gpu)
    m = case.ps["Mass"].astype(np.float64)
    return m[0] * du[0], m[1] * du[1]


def translation(on_gpu):
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=40)
    case.ps["VelocityVec"] = np.tile(np.array([1.3, -0.7], np.float32), (case.n, 1))
    return drho_of(case, on_gpu)


# ------------------------------------------------------------------------------- oracle (CPU)

def test_hydrostatic_interior_oracle():
    assert hydrostatic_interior(False) < 0.01


@pytest.mark.parametrize("dim", [2, 3])
def test_momentum_balance_oracle(dim):
    total, scale = momentum_balance(False, dim)
    assert scale > 0 and total <= 1e-5 * scale


@pytest.mark.parametrize("dim", [2, 3])
def test_two_particle_antisymmetry_oracle(dim):
    fi, fj = two_particles(False, dim)
    assert np.abs(fi).max() > 0
    assert np.abs(fi + fj).max() <= 1e-6 * np.abs(fi).max()


def test_translation_continuity_oracle():
    assert np.all(translation(False) == 0.0)


@pytest.mark.parametrize("kind", KERNELS)
@pytest.mark.parametrize("dim", [2, 3])
def test_kernel_gradient_is_the_derivative(kind, dim):
    h = 0.03
    hinv = 1.0 / h
    eps = 1e-6 * h
    worst, peak = 0.0, 0.0
    for q in np.linspace(0.02, 1.98, 99):
        r = q * h
        _, dw = kernel(kind, dim, r, hinv)
        wp, _ = kernel(kind, dim, r + eps, hinv)
        wm, _ = kernel(kind, dim, r - eps, hinv)
        worst = max(worst, abs(dw - (wp - wm) / (2 * eps)))
        peak = max(peak, abs(dw))
    assert peak > 0 and worst <= 1e-5 * peak, (worst, peak)


# --------------------------------------------------------------------------- CUDA path (GPU)

@pytest.mark.gpu
def test_hydrostatic_interior_gpu():
    assert hydrostatic_interior(True) < 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_momentum_balance_gpu(dim):
    total, scale = momentum_balance(True, dim)
    assert scale > 0 and total <= 1e-5 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_two_particle_antisymmetry_gpu(dim):
    fi, fj = two_particles(True, dim)
    assert np.abs(fi).max() > 0
    assert np.abs(fi + fj).max() <= 1e-6 * np.abs(fi).max()


@pytest.mark.gpu
def test_translation_continuity_gpu():
    assert np.all(translation(True) == 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KERNELS)
@pytest.mark.parametrize("dim", [2, 3])
def test_kernel_gradient_gpu(kind, dim):
    """dW/dr of the CUDA path: particle i moves at 1 m/s straight towards particle j at distance
    r, so its continuity rate is dρ_i/dt = -m_j dW/dr (Continuity.jl:23-34); compared with the
    central difference of W at the same r."""
    h = 0.03
    worst, peak = 0.0, 0.0
    for q in (0.1, 0.4, 0.7, 1.0, 1.3, 1.6, 1.9):
        r = float(np.float32(q * h))
        pos = np.zeros((2, dim))
        pos[1, 0] = r
        vel = np.zeros((2, dim))
        vel[0, 0] = 1.0
        case = tiny_case(pos, vel, [1000.0, 1000.0], h, no_gravity_physics(dim, h, kind))
        drho = drho_of(case, True)
        m_j = float(case.ps["Mass"][1])
        x = case.ps["PositionVec"].astype(np.float64)
        r32 = float(np.linalg.norm(x[1] - x[0]))
        dw_gpu = -drho[0] / m_j * r32 / (x[1, 0] - x[0, 0])
        eps = 1e-6 * h
        wp, _ = kernel(kind, dim, r32 + eps, 1.0 / h)
        wm, _ = kernel(kind, dim, r32 - eps, 1.0 / h)
        fd = (wp - wm) / (2 * eps)
        worst = max(worst, abs(dw_gpu - fd))
        peak = max(peak, abs(fd))
    assert peak > 0 and worst <= 2e-5 * peak, (worst, peak)
