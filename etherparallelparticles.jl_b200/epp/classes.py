"""Host-side mirror of the reference's Class layer for the SPH path.

Same names, argument meaning and errors as the Julia types they mirror:
  Domain2D             src/Class/Domain/Domain2D.jl:10-137 (Float32 cell arithmetic)
  Domain3D             new (the reference's 3D domain is a TODO, AbstractDomain.jl:117-119)
  NamedIndex           src/Class/ParticleSystem/NamedIndex.jl:40-110 (1-based column offsets)
  ActivePair           src/Class/NeighbourSystem/ActivePair.jl:12-33
  NeighbourSystem      src/Class/NeighbourSystem/NeighbourSystem.jl:68-86 (cells live on the device)
  ParticleSystem       src/Class/ParticleSystem/ParticleSystem.jl:28-115 (host matrices are
                       column-major numpy arrays; the device copy is owned by libepp)
"""
import math
from collections import OrderedDict

import numpy as np

from . import abi

f32 = np.float32


class Domain2D:
    """Domain2D{Int32, Float32}(gap, first_x, first_y, last_x, last_y), Domain2D.jl:28-67."""

    dim = 2

    def __init__(self, gap, first_x, first_y, last_x, last_y):
        self.gap = f32(gap)
        self.gap_square = f32(self.gap * self.gap)
        self.first = [f32(first_x), f32(first_y)]
        self.last = [f32(last_x), f32(last_y)]
        self.span = [f32(self.last[a] - self.first[a]) for a in range(2)]
        self.n_axis = [int(math.floor(f32(self.span[a] / self.gap))) for a in range(2)]
        if min(self.n_axis) < 1:
            raise ValueError("domain smaller than one cell")
        self.gap_axis = [f32(self.span[a] / f32(self.n_axis[a])) for a in range(2)]
        self.gap_inv = [f32(f32(1) / self.gap_axis[a]) for a in range(2)]

    # getters of AbstractDomain.jl:28-115
    def get_gap(self): return self.gap
    def get_gap_square(self): return self.gap_square
    def get_n_x(self): return self.n_axis[0]
    def get_n_y(self): return self.n_axis[1]
    def get_n(self): return int(np.prod(self.n_axis))
    def get_first_x(self): return self.first[0]
    def get_first_y(self): return self.first[1]
    def get_last_x(self): return self.last[0]
    def get_last_y(self): return self.last[1]
    def get_span_x(self): return self.span[0]
    def get_span_y(self): return self.span[1]
    def get_gap_x(self): return self.gap_axis[0]
    def get_gap_y(self): return self.gap_axis[1]
    def get_gap_x_inv(self): return self.gap_inv[0]
    def get_gap_y_inv(self): return self.gap_inv[1]

    def _axis(self, a, x):
        i = int(np.floor(f32(f32(f32(x) - self.first[a]) * self.gap_inv[a]))) + 1
        return max(1, min(self.n_axis[a], i))

    def indexCartesianToLinear(self, *ijk):
        lin, stride = 0, 1
        for a, v in enumerate(ijk):
            lin += (v - 1) * stride
            stride *= self.n_axis[a]
        return lin + 1

    def indexLinearToCartesian(self, index):
        out, r = [], index - 1
        for a in range(self.dim):
            out.append(r % self.n_axis[a] + 1)
            r //= self.n_axis[a]
        return tuple(out)

    def inside(self, *x):
        return all(self.first[a] <= f32(x[a]) <= self.last[a] for a in range(self.dim))

    def indexCartesianFromPosition(self, *x):
        return tuple(self._axis(a, x[a]) for a in range(self.dim))

    def indexLinearFromPosition(self, *x):
        return self.indexCartesianToLinear(*self.indexCartesianFromPosition(*x))

    def to_abi(self):
        first = [float(v) for v in self.first] + [0.0] * (3 - self.dim)
        last = [float(v) for v in self.last] + [0.0] * (3 - self.dim)
        return abi.make_domain(self.dim, float(self.gap), first, last)


class Domain3D(Domain2D):
    """3D counterpart of Domain2D with the same Float32 arithmetic (no reference type exists)."""

    dim = 3

    def __init__(self, gap, first_x, first_y, first_z, last_x, last_y, last_z):
        self.gap = f32(gap)
        self.gap_square = f32(self.gap * self.gap)
        self.first = [f32(first_x), f32(first_y), f32(first_z)]
        self.last = [f32(last_x), f32(last_y), f32(last_z)]
        self.span = [f32(self.last[a] - self.first[a]) for a in range(3)]
        self.n_axis = [int(math.floor(f32(self.span[a] / self.gap))) for a in range(3)]
        if min(self.n_axis) < 1:
            raise ValueError("domain smaller than one cell")
        self.gap_axis = [f32(self.span[a] / f32(self.n_axis[a])) for a in range(3)]
        self.gap_inv = [f32(f32(1) / self.gap_axis[a]) for a in range(3)]

    def get_n_z(self): return self.n_axis[2]
    def get_first_z(self): return self.first[2]
    def get_last_z(self): return self.last[2]


class NamedIndexTable:
    """NamedIndexTable, NamedIndex.jl:40-91: 1-based start column per name."""

    def __init__(self, capacity):
        if len(capacity) == 0:
            raise ValueError("empty named tuple")
        self.capacity = OrderedDict((k, int(v)) for k, v in capacity.items())
        self.index = OrderedDict()
        start = 1
        for k, v in self.capacity.items():
            self.index[k] = start
            start += v
        self.n_capacity = start - 1


class NamedIndex:
    """NamedIndex, NamedIndex.jl:95-110."""

    def __init__(self, int_named_tuple, float_named_tuple):
        self.int_table = NamedIndexTable(int_named_tuple)
        self.float_table = NamedIndexTable(float_named_tuple)
        self.combined = OrderedDict(self.int_table.index)
        self.combined.update(self.float_table.index)

    def get_n_int_capacity(self): return self.int_table.n_capacity
    def get_n_float_capacity(self): return self.float_table.n_capacity


# BasicIndex.jl:10-18
kBasicIndexMapDict = {
    "IsMovable": "IsMovable",
    "PositionVec": "PositionVec",
    "Tag": "Tag",
    "nCount": "nCount",
    "nIndex": "nIndex",
    "nRVec": "nRVec",
    "nR": "nR",
}


def mapBasicIndex(named_index_tuple, basic_index_map_dict=None):
    """mapBasicIndex, BasicIndex.jl:20-44 (asserts every basic name resolves)."""
    m = dict(kBasicIndexMapDict)
    if basic_index_map_dict:
        for k in m:
            if k in basic_index_map_dict:
                m[k] = basic_index_map_dict[k]
    out = OrderedDict()
    for k, v in m.items():
        if v not in named_index_tuple:
            raise AssertionError("basic index %s -> %s missing" % (k, v))
        out[k] = named_index_tuple[v]
    return out


class ActivePair:
    """ActivePair, ActivePair.jl:17-33: tag x tag adjacency from a list of pairs."""

    def __init__(self, pair_vector):
        self.pair_vector = [(int(a), int(b)) for a, b in pair_vector]
        maximum_tag = 1
        for a, b in self.pair_vector:
            maximum_tag = max(maximum_tag, a, b)
        self.adjacency_matrix = np.zeros((maximum_tag, maximum_tag), dtype=np.int32)
        for a, b in self.pair_vector:
            self.adjacency_matrix[a - 1, b - 1] = 1


class NeighbourSystem:
    """NeighbourSystem(parallel, domain, active_pair, periodic; max_neighbour_number).

    The reference allocates fixed-capacity cell buckets here (NeighbourSystemBase.jl:76-103).
    The B200 path keeps a counting-sorted cell list on the device instead, so this object only
    records the configuration that the device context is created with.
    """

    def __init__(self, domain, active_pair, periodic_boundary_policy=None,
                 max_neighbour_number=50, max_cell_particles=0):
        if periodic_boundary_policy not in (None, "none", "NonePeriodicBoundaryPolicy"):
            raise NotImplementedError("periodic boundaries are unfinished in the reference "
                                      "(PeriodicBoundary.jl:57) and not supported")
        self.domain = domain
        self.active_pair = active_pair if isinstance(active_pair, ActivePair) else ActivePair(active_pair)
        self.max_neighbour_number = int(max_neighbour_number)
        self.max_cell_particles = int(max_cell_particles)

    def get_n(self):
        return self.domain.get_n()

    def neighbour_cell_counts(self):
        """Counts of the 3^dim stencil, as device_initializeNeighbourSystem! (NeighbourSystemBase.jl:28-48)."""
        n = self.domain.n_axis
        dim = self.domain.dim
        idx = np.indices(n[::-1]).reshape(dim, -1)[::-1]  # x fastest
        cnt = np.ones(idx.shape[1], dtype=np.int32)
        for a in range(dim):
            c = idx[a]
            per = np.where((c == 0) | (c == n[a] - 1), 2, 3) if n[a] > 1 else np.ones_like(c)
            cnt *= per.astype(np.int32)
        return cnt


def defaultCapacityExpand(n):
    return n


class ParticleSystem:
    """Host particle matrices in the reference layout (ParticleSystem.jl:46-115).

    int_properties / float_properties are Fortran-ordered (column-major) numpy arrays of shape
    (n_capacity, n_int_capacity) and (n_capacity, n_float_capacity).  Column offsets are 1-based
    in `named_index` / `basic_index` / `parameters` exactly as in the reference.
    """

    def __init__(self, domain, n_particles, int_named_tuple, float_named_tuple, basic_parameters,
                 capacityExpand=defaultCapacityExpand, basic_index_map_dict=None):
        self.domain = domain
        self.dim = domain.dim
        self.n_particles = int(n_particles)
        self.n_capacity = int(capacityExpand(self.n_particles))
        self.named_index = NamedIndex(int_named_tuple, float_named_tuple)
        self.basic_index = mapBasicIndex(self.named_index.combined, basic_index_map_dict)
        self.basic_parameters = OrderedDict(basic_parameters)
        self.parameters = OrderedDict(self.basic_parameters)
        self.parameters.update(self.named_index.combined)
        self.is_alive = np.zeros(self.n_capacity, dtype=np.int32)
        self.is_alive[: self.n_particles] = 1
        self.cell_index = np.zeros(self.n_capacity, dtype=np.int32)
        self.int_properties = np.zeros(
            (self.n_capacity, self.named_index.get_n_int_capacity()), dtype=np.int32, order="F")
        self.float_properties = np.zeros(
            (self.n_capacity, self.named_index.get_n_float_capacity()), dtype=np.float32, order="F")

    def get_n_particles(self): return self.n_particles
    def get_n_capacity(self): return self.n_capacity
    def get_alive_n_particles(self): return int(self.is_alive.sum())
    def get_n_int_capacity(self): return self.named_index.get_n_int_capacity()
    def get_n_float_capacity(self): return self.named_index.get_n_float_capacity()

    def set_n_particles(self, n):
        self.n_particles = int(n)

    def _col(self, name):
        if name in self.named_index.int_table.index:
            return self.int_properties, self.named_index.int_table.index[name], \
                self.named_index.int_table.capacity[name]
        if name in self.named_index.float_table.index:
            return self.float_properties, self.named_index.float_table.index[name], \
                self.named_index.float_table.capacity[name]
        raise KeyError(name)

    def __getitem__(self, name):
        m, start, width = self._col(name)
        n = self.n_particles
        if width == 1:
            return m[:n, start - 1].copy()
        return m[:n, start - 1: start - 1 + width].copy()

    def __setitem__(self, name, value):
        m, start, width = self._col(name)
        n = self.n_particles
        if width == 1:
            m[:n, start - 1] = value
        else:
            m[:n, start - 1: start - 1 + width] = value

    def column_map(self, names=None):
        """epp_column_map (0-based) from the reference's property names and aliases.

        The reference names come from src/SPH/Macro/Scalar.jl:11-33 and Vector.jl:11-18 and the
        basic index (BasicIndex.jl:10-18); names absent from the named tuples map to -1."""
        names = names or {}
        lookup = {
            "tag": "Tag", "is_movable": "IsMovable", "n_count": "nCount", "n_index": "nIndex",
            "position": "PositionVec", "velocity": "VelocityVec", "dvelocity": "dVelocityVec",
            "mass": "Mass", "volume": "Volume", "density": "Density", "ddensity": "dDensity",
            "pressure": "Pressure", "gap": "Gap", "h": "H", "n_rvec": "nRVec", "n_r": "nR",
            "n_w": "nW", "n_dw": "nDW", "n_hinv": "nHInv", "instance": "Instance",
        }
        m = abi.epp_column_map.empty()
        for field, ref in lookup.items():
            ref = names.get(field, ref)
            if ref in self.basic_index and field in ("tag", "is_movable", "n_count", "n_index",
                                                     "position", "n_rvec", "n_r"):
                setattr(m, field, self.basic_index[ref] - 1)
            elif ref in self.named_index.int_table.index:
                setattr(m, field, self.named_index.int_table.index[ref] - 1)
            elif ref in self.named_index.float_table.index:
                setattr(m, field, self.named_index.float_table.index[ref] - 1)
        return m
