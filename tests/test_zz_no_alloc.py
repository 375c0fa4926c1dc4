"""epp_cell_sort_noalloc: the cell-list build for callers that cannot allocate device memory.

Some hosts drive the library from code that must not call cudaMalloc -- an application that owns a
fixed device pool, or a loop in the middle of a step where an allocation would synchronise the
device.  This entry point keeps its intermediate arrays in a static device array of the library
and works on buffers the caller passes in.  The test checks it against the context path
(epp_search + epp_cell_stats) and against the oracle's cell list on two calls in a row, since
every call reuses that same array.
The buffers below are the caller's (the test allocates them with torch); the entry point itself
allocates nothing.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from epp import abi, casegen
from epp import lib as epplib
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem

pytestmark = pytest.mark.gpu


def _context_cells(case, pos):
    """Counts, offsets and sorted ids from the existing entry points (epp_search + epp_cell_stats)."""
    ps = case.ps
    ps["PositionVec"] = pos
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    d = DeviceParticleSystem(ps, ns)
    d.syncto()
    d.ctx.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_NONE, case.physics, 0)
    d.ctx.synchronize(raise_on_status=False)
    out = d.ctx.cell_stats()
    d.close()
    return out


def _oracle_cells(case, pos):
    """Counts, offsets and sorted ids of the oracle's bucket insert (NeighbourSearch.jl:12-47)."""
    from helpers import config_for
    from oracle_lib import Oracle
    ps = case.ps
    ps["PositionVec"] = pos
    ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
    o = Oracle(config_for(ps, ns, max_cell_particles=64 if case.meta["dim"] == 2 else 128), 32)
    o.upload(ps.n_particles, ps.is_alive, ps.cell_index, ps.int_properties, ps.float_properties, ps.column_map())
    o.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_NONE, case.physics)
    oc, oo, oi = o.cell_stats(ps.n_particles)   # ids buffer sized for every particle
    return oc, oo, oi[: int(oo[-1])]


def _noalloc(domain, pos):
    import torch
    lib = epplib.load()
    n = pos.shape[0]
    dim = pos.shape[1]
    n_cells = domain.get_n()
    dpos = torch.from_numpy(np.ascontiguousarray(pos.T).reshape(-1)).cuda()   # column-major
    counts = torch.full((n_cells,), -1, dtype=torch.int32, device="cuda")
    offsets = torch.full((n_cells + 1,), -1, dtype=torch.int32, device="cuda")
    ids = torch.zeros((max(n, 1),), dtype=torch.int32, device="cuda")
    n_alive = C.c_int32(-1)
    dom = domain.to_abi()
    torch.cuda.synchronize()
    rc = lib.epp_cell_sort_noalloc(C.byref(dom), n, C.c_void_p(dpos.data_ptr()), C.c_void_p(counts.data_ptr()),
                                   C.c_void_p(offsets.data_ptr()), C.c_void_p(ids.data_ptr()),
                                   C.byref(n_alive), None)
    assert rc == abi.EPP_OK, abi.STATUS_NAMES.get(rc, rc)
    assert dim == domain.dim
    return counts.cpu().numpy(), offsets.cpu().numpy(), ids.cpu().numpy()[: n_alive.value], n_alive.value


@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_matches_context_path_twice(dim):
    if dim == 2:
        case = casegen.dam_break_2d(dx=0.02, max_neighbour_number=1)
    else:
        case = casegen.dam_break_3d(dx=0.02, tank=(0.6, 0.3, 0.4), column=(0.2, 0.3, 0.24), max_neighbour_number=1)
    rng = np.random.default_rng(7)
    pos0 = case.ps["PositionVec"].astype(np.float32)
    for call in range(2):
        # a different arrangement per call, with a few particles outside the domain (dropped)
        pos = pos0 + rng.normal(0, 0.3 * case.meta["dx"], pos0.shape).astype(np.float32)
        pos[:: 97] = 1e3
        rc, ro, ri = _context_cells(case, pos)
        c, o, ids, n_alive = _noalloc(case.domain, pos)
        assert n_alive == int(ro[-1])
        assert np.array_equal(c, rc), "counts differ on call %d" % call
        assert np.array_equal(o, ro), "offsets differ on call %d" % call
        assert np.array_equal(ids, ri), "sorted ids differ on call %d" % call
        # and the oracle's cell list of the same positions
        oc, oo, oi = _oracle_cells(case, pos)
        assert np.array_equal(c, oc) and np.array_equal(o, oo) and np.array_equal(ids, oi), \
            "the oracle's cell list differs on call %d" % call


def test_noalloc_rejects_oversize():
    lib = epplib.load()
    mp, mc, sb = C.c_int32(), C.c_int32(), C.c_int64()
    lib.epp_noalloc_limits(C.byref(mp), C.byref(mc), C.byref(sb))
    n_alive = C.c_int32()
    d = abi.make_domain(2, 0.1, [0.0, 0.0], [1.0, 1.0])
    rc = lib.epp_cell_sort_noalloc(C.byref(d), mp.value + 1, C.c_void_p(16), None, None, C.c_void_p(16),
                                   C.byref(n_alive), None)
    assert rc == abi.EPP_ERR_CAPACITY
    big = abi.make_domain(2, 1e-4, [0.0, 0.0], [1.0, 1.0])   # 10^8 cells
    rc = lib.epp_cell_sort_noalloc(C.byref(big), 10, C.c_void_p(16), None, None, C.c_void_p(16),
                                   C.byref(n_alive), None)
    assert rc == abi.EPP_ERR_CAPACITY
