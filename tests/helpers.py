"""Shared test helpers: build configs from the host mirror and the golden fixtures."""
import json
import os
from collections import OrderedDict

import numpy as np

from epp import abi
from epp.classes import Domain2D, NeighbourSystem, ParticleSystem

HERE = os.path.dirname(os.path.abspath(__file__))


def kat():
    with open(os.path.join(HERE, "golden", "reference_kat.json")) as f:
        return json.load(f)


def config_for(ps, ns, hbm_budget_bytes=0, max_cell_particles=0):
    adj = ns.active_pair.adjacency_matrix.tolist()
    return abi.make_config(ps.domain.to_abi(), ps.n_capacity, adj,
                           max_neighbour_number=ns.max_neighbour_number,
                           max_cell_particles=max_cell_particles,
                           hbm_budget_bytes=hbm_budget_bytes)


def nine_particle_system():
    """The 9-particle case of test/Algorithm/NeighbourSearchTest.jl:11-66."""
    k = kat()["neighbour_search"]
    d = k["domain"]
    domain = Domain2D(d["gap"], d["first"][0], d["first"][1], d["last"][0], d["last"][1])
    nb = k["max_neighbour_number"]
    ints = OrderedDict([("Tag", 1), ("IsMovable", 1), ("nCount", 1), ("nIndex", nb)])
    floats = OrderedDict([("RVec", 2), ("nRVec", 2 * nb), ("nR", nb), ("dVelocityVec", 2)])
    ps = ParticleSystem(domain, 9, ints, floats, OrderedDict([("c_0", 340.0), ("gamma", 7), ("mu", 1e-3)]),
                        basic_index_map_dict={"PositionVec": "RVec", "nCount": "nCount",
                                              "nIndex": "nIndex", "nR": "nR"})
    ps["RVec"] = np.array(k["positions"], dtype=np.float32)
    ps["Tag"] = np.array(k["tags"], dtype=np.int32)
    ns = NeighbourSystem(domain, [tuple(p) for p in k["active_pair"]], max_neighbour_number=nb)
    return ps, ns, k


def neighbour_sets(ps):
    """Sorted 1-based neighbour ids per particle from the host matrices."""
    bi = ps.basic_index
    out = []
    for i in range(ps.n_particles):
        c = ps.int_properties[i, bi["nCount"] - 1]
        out.append(sorted(ps.int_properties[i, bi["nIndex"] - 1: bi["nIndex"] - 1 + c].tolist()))
    return out
