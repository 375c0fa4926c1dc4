"""Dam-break case generator (2D and 3D) in the reference layout.

Restates example/collapse_dry/same/casegen.jl:17-146 and Geometry.create(::Rectangle)
(src/Geometry/Geometry2D.jl:71-101) with the benchmark physics: hydrostatic initial density,
Tait EOS, c0 = 10 sqrt(2 g H), h = 1.5 dx (2D) / 1.3 dx (3D), cell gap 2h, dt = 0.1 h / c0.

`reference_quirk=True` reproduces Geometry2D.jl:83, which uses mod(i, n_x) where mod1 is meant,
so the last particle of every lattice row lands at first_x - 0.5 dx.  The default is the
intended lattice.  The 3D generator has no reference counterpart (Geometry3D.jl:89-94 is a stub).
"""
import math
from collections import OrderedDict

import numpy as np

from . import abi
from .classes import Domain2D, Domain3D, ParticleSystem

FLUID_TAG = 1
WALL_TAG = 2
RHO0 = 1000.0
GRAVITY = 9.81
GAMMA = 7


def lattice(first, last, gap, reference_quirk=False):
    """Cell-centred lattice over an axis-aligned box; returns (positions float32 (n, dim), volume, gap).

    2D follows Geometry.create(::Rectangle): n_a = round(span_a / gap), d_a = span_a / n_a,
    volume = prod(d_a), particle gap = sqrt(prod) (cube root in 3D)."""
    dim = len(first)
    first = [np.float32(v) for v in first]
    last = [np.float32(v) for v in last]
    span = [np.float32(last[a] - first[a]) for a in range(dim)]
    n = [int(round(float(span[a]) / gap)) for a in range(dim)]
    d = [np.float32(span[a] / np.float32(n[a])) for a in range(dim)]
    volume = float(np.prod([float(v) for v in d]))
    pgap = volume ** (1.0 / dim)
    total = int(np.prod(n))
    i = np.arange(1, total + 1, dtype=np.int64)
    idx = []
    r = i - 1
    for a in range(dim):
        if a == 0:
            ia = (i % n[0]) if reference_quirk else ((i - 1) % n[0] + 1)
        else:
            ia = r % n[a] + 1
        idx.append(ia)
        r = r // n[a]
    pos = np.empty((total, dim), dtype=np.float32)
    for a in range(dim):
        pos[:, a] = (np.float64(first[a]) + (idx[a] - 0.5) * np.float64(d[a])).astype(np.float32)
    return pos, np.float32(volume), np.float32(pgap)


def tait_b(rho0, c0, gamma):
    return rho0 * c0 * c0 / gamma


def hydrostatic_density(y, height, rho0, c0, g=GRAVITY, gamma=GAMMA):
    """rho(y) with p = rho0 g (H - y) on the Tait EOS: rho0 (1 + rho0 g (H - y) / B)^(1/gamma)."""
    B = tait_b(rho0, c0, gamma)
    return rho0 * np.power(1.0 + rho0 * g * (height - y) / B, 1.0 / gamma)


class DamBreakCase:
    """A generated case: particle system (host, reference layout), domain, physics and metadata."""

    def __init__(self, ps, domain, physics, meta):
        self.ps = ps
        self.domain = domain
        self.physics = physics
        self.meta = meta

    @property
    def n(self):
        return self.ps.n_particles


def _layout(dim, max_nb):
    ints = OrderedDict([("Tag", 1), ("IsMovable", 1), ("nCount", 1), ("nIndex", max_nb)])
    floats = OrderedDict([
        ("PositionVec", dim), ("VelocityVec", dim), ("dVelocityVec", dim), ("AccelerationVec", dim),
        ("Mass", 1), ("Volume", 1), ("Density", 1), ("dDensity", 1), ("Pressure", 1), ("Gap", 1),
        ("H", 1), ("SumWeight", 1), ("SumWeightedDensity", 1), ("SumWeightedPressure", 1),
        ("nW", max_nb), ("nDW", max_nb), ("nHInv", max_nb), ("nRVec", max_nb * dim), ("nR", max_nb),
    ])
    return ints, floats


def dam_break_2d(dx=0.02, tank=(4.0, 3.0), column=(1.0, 2.0), wall_layers=3, h_factor=1.5,
                 max_neighbour_number=40, reference_quirk=False, kahan=1,
                 viscosity=abi.EPP_VISCOSITY_REFERENCE, alpha=0.1, beta=0.1):
    """2D dry dam break (casegen.jl:17-146 geometry; benchmark physics)."""
    x0, y0 = 0.0, 0.0
    ww = wall_layers * dx
    h = h_factor * dx
    gap = 2.0 * h
    height = column[1]
    c0 = 10.0 * math.sqrt(2.0 * GRAVITY * height)
    domain = Domain2D(gap, x0 - ww, y0 - ww, x0 + tank[0] + ww, y0 + tank[1] + ww)
    parts = []
    fp, fv, fg = lattice([x0, y0], [x0 + column[0], y0 + column[1]], dx, reference_quirk)
    parts.append((fp, fv, fg, FLUID_TAG, 1))
    for lo, hi in [
        ([x0 - ww, y0 - ww], [x0 + tank[0] + ww, y0]),      # bottom
        ([x0 - ww, y0], [x0, y0 + tank[1]]),                # left
        ([x0 + tank[0], y0], [x0 + tank[0] + ww, y0 + tank[1]]),  # right
    ]:
        wp, wv, wg = lattice(lo, hi, dx, reference_quirk)
        parts.append((wp, wv, wg, WALL_TAG, 0))
    return _assemble(2, domain, parts, h_factor, height, c0, max_neighbour_number, kahan,
                     viscosity, alpha, beta, {"dx": dx, "tank": tank, "column": column,
                                              "reference_quirk": reference_quirk})


def dam_break_3d(dx=0.005, tank=(3.2, 1.0, 1.0), column=(1.0, 1.0, 0.6), wall_layers=3,
                 h_factor=1.3, max_neighbour_number=1, kahan=1,
                 viscosity=abi.EPP_VISCOSITY_REFERENCE, alpha=0.1, beta=0.1):
    """3D dam break: water block in a box tank with 3-layer floor and side walls (z is up).

    The reference has no 3D path; this is the natural extension of the 2D case."""
    ww = wall_layers * dx
    h = h_factor * dx
    gap = 2.0 * h
    height = column[2]
    c0 = 10.0 * math.sqrt(2.0 * GRAVITY * height)
    L, W, Ht = tank
    domain = Domain3D(gap, -ww, -ww, -ww, L + ww, W + ww, Ht + ww)
    parts = []
    fp, fv, fg = lattice([0.0, 0.0, 0.0], list(column), dx)
    parts.append((fp, fv, fg, FLUID_TAG, 1))
    for lo, hi in [
        ([-ww, -ww, -ww], [L + ww, W + ww, 0.0]),   # floor
        ([-ww, 0.0, 0.0], [0.0, W, Ht]),             # x- wall
        ([L, 0.0, 0.0], [L + ww, W, Ht]),            # x+ wall
        ([0.0, -ww, 0.0], [L, 0.0, Ht]),             # y- wall
        ([0.0, W, 0.0], [L, W + ww, Ht]),            # y+ wall
    ]:
        wp, wv, wg = lattice(lo, hi, dx)
        parts.append((wp, wv, wg, WALL_TAG, 0))
    return _assemble(3, domain, parts, h_factor, height, c0, max_neighbour_number, kahan,
                     viscosity, alpha, beta, {"dx": dx, "tank": tank, "column": column})


def _assemble(dim, domain, parts, h_factor, height, c0, max_nb, kahan, viscosity, alpha, beta, meta):
    n = sum(p[0].shape[0] for p in parts)
    ints, floats = _layout(dim, max_nb)
    params = OrderedDict([("rho0", RHO0), ("p0", 0.0), ("FLUID_TAG", FLUID_TAG),
                          ("WALL_TAG", WALL_TAG), ("gap0", meta["dx"]),
                          ("h0", h_factor * meta["dx"])])
    ps = ParticleSystem(domain, n, ints, floats, params)
    pos = np.concatenate([p[0] for p in parts])
    vol = np.concatenate([np.full(p[0].shape[0], p[1], np.float32) for p in parts])
    pg = np.concatenate([np.full(p[0].shape[0], p[2], np.float32) for p in parts])
    tag = np.concatenate([np.full(p[0].shape[0], p[3], np.int32) for p in parts])
    mov = np.concatenate([np.full(p[0].shape[0], p[4], np.int32) for p in parts])
    up = dim - 1
    rho = np.full(n, RHO0, np.float64)
    fl = tag == FLUID_TAG
    rho[fl] = hydrostatic_density(pos[fl, up].astype(np.float64), height, RHO0, c0)
    rho = rho.astype(np.float32)
    B = tait_b(RHO0, c0, GAMMA)
    p = (B * ((rho.astype(np.float64) / RHO0) ** GAMMA - 1.0)).astype(np.float32)
    ps["PositionVec"] = pos
    ps["Volume"] = vol
    ps["Gap"] = pg
    ps["Tag"] = tag
    ps["IsMovable"] = mov
    ps["Density"] = rho
    ps["Mass"] = (rho * vol).astype(np.float32)          # Mass = Density .* Volume (casegen.jl:85)
    ps["H"] = (pg * np.float32(h_factor)).astype(np.float32)   # H = Gap * 1.5 (casegen.jl:86)
    ps["Pressure"] = p
    h0 = np.float32(h_factor * meta["dx"])
    c0f = np.float32(c0)
    dt = float(np.float32(0.1 * float(h0) / float(c0f)))   # dt = 0.1 h0 / c0 (main.jl:68)
    grav = (0.0, -GRAVITY, 0.0) if dim == 2 else (0.0, 0.0, -GRAVITY)
    physics = abi.make_physics(dt, rho0=RHO0, c0=float(c0f), p0=0.0, gamma=GAMMA, gravity=grav,
                               alpha=alpha, beta=beta, viscosity=viscosity, fluid_tag=FLUID_TAG,
                               wall_tag=WALL_TAG, kahan=kahan)
    meta = dict(meta)
    meta.update({"n": n, "n_fluid": int(fl.sum()), "n_wall": int((~fl).sum()), "c0": float(c0f),
                 "dt": dt, "h": float(h0), "dim": dim, "height": height,
                 "n_cells": domain.get_n()})
    return DamBreakCase(ps, domain, physics, meta)


# active pairs of casegen.jl:137: fluid-fluid, fluid-wall, wall-fluid
DAM_BREAK_ACTIVE_PAIRS = [(FLUID_TAG, FLUID_TAG), (FLUID_TAG, WALL_TAG), (WALL_TAG, FLUID_TAG)]
