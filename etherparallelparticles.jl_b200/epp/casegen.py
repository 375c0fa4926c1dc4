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


def _layout(dim, max_nb, instance=False):
    ints = OrderedDict([("Tag", 1), ("IsMovable", 1), ("nCount", 1), ("nIndex", max_nb)])
    if instance:
        ints["Instance"] = 1   # batch: 0-based instance of the particle (no reference counterpart)
    floats = OrderedDict([
        ("PositionVec", dim), ("VelocityVec", dim), ("dVelocityVec", dim), ("AccelerationVec", dim),
        ("Mass", 1), ("Volume", 1), ("Density", 1), ("dDensity", 1), ("Pressure", 1), ("Gap", 1),
        ("H", 1), ("SumWeight", 1), ("SumWeightedDensity", 1), ("SumWeightedPressure", 1),
        ("nW", max_nb), ("nDW", max_nb), ("nHInv", max_nb), ("nRVec", max_nb * dim), ("nR", max_nb),
    ])
    return ints, floats


def dam_break_2d(dx=0.02, tank=(4.0, 3.0), column=(1.0, 2.0), wall_layers=3, h_factor=1.5,
                 max_neighbour_number=40, reference_quirk=False, kahan=1,
                 viscosity=abi.EPP_VISCOSITY_REFERENCE, alpha=0.1, beta=0.1, physics="benchmark"):
    """2D dry dam break (casegen.jl:17-146 geometry).  physics="benchmark": Wendland C2, Tait EOS,
    artificial viscosity, symplectic Euler, hydrostatic initial density.  physics="example": the
    reference example's own (main.jl:53-144): CubicSpline, linear EOS with c0 = 120, classic
    viscosity mu = 1e-3, sAccelerateMove!, kernel filter every 20 steps, g = 9.8,
    dt = 2 * 0.1 h0 / c0, uniform initial density rho0 and pressure p0."""
    height = column[1]
    c0 = 10.0 * math.sqrt(2.0 * GRAVITY * height)
    domain = _tank_domain_2d(dx, tank, wall_layers, h_factor)
    parts = _dam_parts_2d(dx, tank, column, wall_layers, reference_quirk)
    if physics == "example":
        return _assemble_example(domain, parts, h_factor, max_neighbour_number,
                                 {"dx": dx, "tank": tank, "column": column, "reference_quirk": reference_quirk})
    return _assemble(2, domain, parts, h_factor, height, c0, max_neighbour_number, kahan,
                     viscosity, alpha, beta, {"dx": dx, "tank": tank, "column": column,
                                              "reference_quirk": reference_quirk})


EXAMPLE_C0 = 120.0    # main.jl:57
EXAMPLE_MU0 = 1e-3    # casegen.jl:78
EXAMPLE_G = 9.8       # main.jl:56


def _assemble_example(domain, parts, h_factor, max_nb, meta):
    st = _state(2, parts, h_factor, 1.0, EXAMPLE_C0)
    n = st["Tag"].shape[0]
    st["Density"] = np.full(n, np.float32(RHO0), np.float32)          # casegen.jl:93,103
    st["Mass"] = (st["Density"] * st["Volume"]).astype(np.float32)
    st["Pressure"] = np.zeros(n, np.float32)                          # p0 = 0
    ints, floats = _layout(2, max_nb)
    params = OrderedDict([("rho0", RHO0), ("p0", 0.0), ("FLUID_TAG", FLUID_TAG), ("WALL_TAG", WALL_TAG),
                          ("gap0", meta["dx"]), ("h0", h_factor * meta["dx"]), ("mu0", EXAMPLE_MU0)])
    ps = ParticleSystem(domain, n, ints, floats, params)
    for k, v in st.items():
        ps[k] = v
    h0 = np.float32(h_factor * meta["dx"])
    c0f = np.float32(EXAMPLE_C0)
    dt = float(np.float32(np.float32(0.1 * float(h0) / float(c0f))) * np.float32(2))   # main.jl:68
    physics = abi.make_physics(dt, rho0=RHO0, c0=float(c0f), p0=0.0, gamma=GAMMA, gravity=(0.0, -EXAMPLE_G, 0.0),
                               alpha=0.0, beta=0.0, viscosity=abi.EPP_VISCOSITY_CLASSIC, fluid_tag=FLUID_TAG,
                               wall_tag=WALL_TAG, kahan=0, kernel=abi.EPP_KERNEL_CUBIC_SPLINE,
                               eos=abi.EPP_EOS_LINEAR, mu=EXAMPLE_MU0, motion=abi.EPP_MOTION_ACCELERATE_MOVE,
                               filter_interval=20)
    fl = st["Tag"] == FLUID_TAG
    meta = dict(meta)
    meta.update({"n": n, "n_fluid": int(fl.sum()), "n_wall": int((~fl).sum()), "c0": float(c0f), "dt": dt,
                 "h": float(h0), "dim": 2, "height": meta["column"][1], "n_cells": domain.get_n(),
                 "physics": "example"})
    return DamBreakCase(ps, domain, physics, meta)


def _tank_domain_2d(dx, tank, wall_layers, h_factor):
    ww = wall_layers * dx
    return Domain2D(2.0 * h_factor * dx, -ww, -ww, tank[0] + ww, tank[1] + ww)


def _dam_parts_2d(dx, tank, column, wall_layers, reference_quirk=False):
    """Fluid column at the tank's lower-left corner and 3-layer floor and side walls."""
    x0, y0 = 0.0, 0.0
    ww = wall_layers * dx
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
    return parts


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


def _state(dim, parts, h_factor, height, c0):
    """Per-particle initial state of one case: hydrostatic density on the Tait EOS with this
    case's c0 and column height, Mass = Density .* Volume, H = Gap * h_factor."""
    n = sum(p[0].shape[0] for p in parts)
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
    return {"PositionVec": pos, "Volume": vol, "Gap": pg, "Tag": tag, "IsMovable": mov, "Density": rho,
            "Mass": (rho * vol).astype(np.float32),            # Mass = Density .* Volume (casegen.jl:85)
            "H": (pg * np.float32(h_factor)).astype(np.float32),  # H = Gap * 1.5 (casegen.jl:86)
            "Pressure": p}


def _time_step(h_factor, dx, c0):
    """(float32 c0, dt = 0.1 h0 / c0 (main.jl:68) rounded to float32)."""
    h0 = np.float32(h_factor * dx)
    c0f = np.float32(c0)
    return float(c0f), float(np.float32(0.1 * float(h0) / float(c0f)))


def _physics(dim, dt, c0, kahan, viscosity, alpha, beta):
    grav = (0.0, -GRAVITY, 0.0) if dim == 2 else (0.0, 0.0, -GRAVITY)
    return abi.make_physics(dt, rho0=RHO0, c0=c0, p0=0.0, gamma=GAMMA, gravity=grav,
                            alpha=alpha, beta=beta, viscosity=viscosity, fluid_tag=FLUID_TAG,
                            wall_tag=WALL_TAG, kahan=kahan)


def _assemble(dim, domain, parts, h_factor, height, c0, max_nb, kahan, viscosity, alpha, beta, meta):
    st = _state(dim, parts, h_factor, height, c0)
    n = st["Tag"].shape[0]
    ints, floats = _layout(dim, max_nb)
    params = OrderedDict([("rho0", RHO0), ("p0", 0.0), ("FLUID_TAG", FLUID_TAG),
                          ("WALL_TAG", WALL_TAG), ("gap0", meta["dx"]),
                          ("h0", h_factor * meta["dx"])])
    ps = ParticleSystem(domain, n, ints, floats, params)
    for k, v in st.items():
        ps[k] = v
    c0f, dt = _time_step(h_factor, meta["dx"], c0)
    physics = _physics(dim, dt, c0f, kahan, viscosity, alpha, beta)
    fl = st["Tag"] == FLUID_TAG
    meta = dict(meta)
    meta.update({"n": n, "n_fluid": int(fl.sum()), "n_wall": int((~fl).sum()), "c0": c0f,
                 "dt": dt, "h": float(np.float32(h_factor * meta["dx"])), "dim": dim, "height": height,
                 "n_cells": domain.get_n()})
    return DamBreakCase(ps, domain, physics, meta)


class BatchCase(DamBreakCase):
    """Independent instances in one particle system (an Instance column), with per-instance
    time step and speed of sound (`inst_dt`, `inst_c0`) and each instance's particle rows."""

    def __init__(self, ps, domain, physics, meta, inst_dt, inst_c0, rows):
        super().__init__(ps, domain, physics, meta)
        self.inst_dt = inst_dt
        self.inst_c0 = inst_c0
        self.rows = rows   # rows[k] = (first, last + 1) of instance k in the particle matrices

    @property
    def n_instances(self):
        return len(self.rows)


def batch_columns(n_instances, seed=0, width=(0.5, 1.5), height=(1.0, 2.5)):
    """The seeded column sizes of a batch: width ~ U[width], height ~ U[height] per instance."""
    rng = np.random.default_rng(seed)
    w = rng.uniform(width[0], width[1], n_instances)
    h = rng.uniform(height[0], height[1], n_instances)
    return [(float(a), float(b)) for a, b in zip(w, h)]


def dam_break_batch(n_instances=256, seed=0, dx=0.01, tank=(4.0, 3.0), width=(0.5, 1.5),
                    height=(1.0, 2.5), wall_layers=3, h_factor=1.5, max_neighbour_number=1, kahan=1,
                    viscosity=abi.EPP_VISCOSITY_REFERENCE, alpha=0.1, beta=0.1, columns=None):
    """Uneven 2D dam breaks in one batch: instance k is dam_break_2d(dx, tank, columns[k]) --
    the same particles, state and physics as that case built alone -- with c0_k = 10 sqrt(2 g H_k)
    and dt_k = 0.1 h / c0_k of its own column height."""
    columns = columns or batch_columns(n_instances, seed, width, height)
    domain = _tank_domain_2d(dx, tank, wall_layers, h_factor)
    states, inst_dt, inst_c0, rows, n_fluid = [], [], [], [], []
    first = 0
    for (w, hgt) in columns:
        c0 = 10.0 * math.sqrt(2.0 * GRAVITY * hgt)
        st = _state(2, _dam_parts_2d(dx, tank, (w, hgt), wall_layers), h_factor, hgt, c0)
        c0f, dt = _time_step(h_factor, dx, c0)
        states.append(st)
        inst_dt.append(dt)
        inst_c0.append(c0f)
        n = st["Tag"].shape[0]
        rows.append((first, first + n))
        n_fluid.append(int((st["Tag"] == FLUID_TAG).sum()))
        first += n
    ints, floats = _layout(2, max_neighbour_number, instance=True)
    params = OrderedDict([("rho0", RHO0), ("p0", 0.0), ("FLUID_TAG", FLUID_TAG),
                          ("WALL_TAG", WALL_TAG), ("gap0", dx), ("h0", h_factor * dx)])
    ps = ParticleSystem(domain, first, ints, floats, params)
    for k in states[0]:
        ps[k] = np.concatenate([st[k] for st in states])
    ps["Instance"] = np.concatenate([np.full(r[1] - r[0], k, np.int32) for k, r in enumerate(rows)])
    physics = _physics(2, inst_dt[0], inst_c0[0], kahan, viscosity, alpha, beta)
    meta = {"dim": 2, "dx": dx, "tank": tank, "n": first, "n_fluid": int(sum(n_fluid)),
            "n_wall": first - int(sum(n_fluid)), "columns": columns, "seed": seed,
            "inst_n_fluid": n_fluid, "h": float(np.float32(h_factor * dx)),
            "n_cells": domain.get_n() * len(columns)}
    return BatchCase(ps, domain, physics, meta, np.array(inst_dt, np.float32), np.array(inst_c0, np.float32),
                     rows)


def batch_key(case):
    """Cases with equal keys can run as instances of one batch: 2D, the same domain (cell grid)
    and neighbour capacity, and the same physics except each instance's dt and c0."""
    if case.meta.get("dim") != 2 or isinstance(case, BatchCase):
        return None
    d = case.domain
    p = case.physics
    phys = tuple((f, repr(getattr(p, f)[:] if hasattr(getattr(p, f), "__len__") else getattr(p, f)))
                 for f, _ in p._fields_ if f not in ("dt", "c0"))
    nb = case.ps.named_index.int_table.capacity["nIndex"]
    return (2, float(d.gap), tuple(float(v) for v in d.first), tuple(float(v) for v in d.last), nb, phys)


def merge_cases(cases):
    """One BatchCase holding `cases` (equal batch_key) as instances 0..K-1, in order: every
    particle column copied, an Instance column added, each instance keeping its own dt and c0."""
    if not cases:
        raise ValueError("no cases")
    key = batch_key(cases[0])
    if key is None or any(batch_key(c) != key for c in cases):
        raise ValueError("cases differ in domain or physics: they cannot share a batch")
    first = cases[0]
    nb = first.ps.named_index.int_table.capacity["nIndex"]
    ints, floats = _layout(2, nb, instance=True)
    rows, total = [], 0
    for c in cases:
        rows.append((total, total + c.n))
        total += c.n
    ps = ParticleSystem(first.domain, total, ints, floats, OrderedDict(first.ps.basic_parameters))
    for name in list(ints) + list(floats):
        if name == "Instance":
            continue
        ps[name] = np.concatenate([c.ps[name] for c in cases])
    ps["Instance"] = np.concatenate([np.full(c.n, k, np.int32) for k, c in enumerate(cases)])
    meta = dict(first.meta)
    meta.update({"n": total, "n_fluid": int(sum(c.meta["n_fluid"] for c in cases)),
                 "n_wall": int(sum(c.meta["n_wall"] for c in cases)),
                 "inst_n_fluid": [c.meta["n_fluid"] for c in cases],
                 "n_cells": first.domain.get_n() * len(cases)})
    return BatchCase(ps, first.domain, first.physics, meta,
                     np.array([c.physics.dt for c in cases], np.float32),
                     np.array([c.physics.c0 for c in cases], np.float32), rows)


# active pairs of casegen.jl:137: fluid-fluid, fluid-wall, wall-fluid
DAM_BREAK_ACTIVE_PAIRS = [(FLUID_TAG, FLUID_TAG), (FLUID_TAG, WALL_TAG), (WALL_TAG, FLUID_TAG)]
