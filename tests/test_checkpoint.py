"""Checkpoint / resume with the raw writer's datasets (raw/int_properties, raw/float_properties,
appendix/*) in its JLD2 files (and the .npz alternative): an exact round trip of the alive rows on
the host, and (GPU) a run resumed from a checkpoint staying with the uninterrupted run."""
import numpy as np
import pytest

from epp import abi, casegen, checkpoint
from epp.algorithm import DeviceParticleSystem
from epp.classes import NeighbourSystem


@pytest.mark.parametrize("suffix", [".jld2", ".npz"])
def test_round_trip_alive_rows(tmp_path, suffix):
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=8)
    ps = case.ps
    ps["Density"] = np.linspace(990, 1010, ps.n_particles).astype(np.float32)
    ps.is_alive[[3, 10]] = 0
    path = checkpoint.file_name(str(tmp_path), 7, suffix=suffix)
    assert path.endswith("result_0007" + suffix)
    checkpoint.save(ps, path, checkpoint.appendix(step=7, time_value=0.25, write_step=2))
    fresh = casegen.dam_break_2d(dx=0.04, max_neighbour_number=8).ps
    app = checkpoint.load(fresh, path)
    keep = np.ones(ps.n_particles, bool)
    keep[[3, 10]] = False
    assert fresh.n_particles == ps.n_particles - 2
    assert np.array_equal(fresh.int_properties[: fresh.n_particles], ps.int_properties[: ps.n_particles][keep])
    assert np.array_equal(fresh.float_properties[: fresh.n_particles], ps.float_properties[: ps.n_particles][keep])
    assert fresh.is_alive[: fresh.n_particles].all() and not fresh.is_alive[fresh.n_particles:].any()
    assert app["TMSTEP"] == 7 and app["TimeValue"] == 0.25 and app["WriteStep"] == 2 and app["TimeStamp"]


def test_load_rejects_other_layout(tmp_path):
    a = casegen.dam_break_2d(dx=0.04, max_neighbour_number=8)
    path = checkpoint.save(a.ps, str(tmp_path / "c.jld2"))
    b = casegen.dam_break_2d(dx=0.04, max_neighbour_number=40)
    with pytest.raises(ValueError):
        checkpoint.load(b.ps, path)


@pytest.mark.gpu
def test_resume_follows_uninterrupted_run(tmp_path):
    SYM, CONT = abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY

    def system(case):
        ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        d = DeviceParticleSystem(case.ps, ns)
        d.syncto()
        d.ctx.search(SYM, CONT, case.physics, 0)
        return d

    a = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
    phys = a.physics
    da = system(a)
    da.ctx.step(10, phys)
    da.asyncto()
    path = checkpoint.save(a.ps, checkpoint.file_name(str(tmp_path), 10), checkpoint.appendix(step=10))
    da.ctx.step(10, phys)
    da.asyncto()
    b = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
    app = checkpoint.load(b.ps, path)
    assert app["TMSTEP"] == 10
    # the restart's search! adds the continuity rate to dDensity (as the reference's search action
    # does), so the saved rate is cleared first
    checkpoint.prepare_restart(b.ps)
    db = system(b)
    db.ctx.step(10, phys)
    db.asyncto()
    xa, xb = a.ps["PositionVec"], b.ps["PositionVec"]
    assert np.max(np.abs(xa - xb)) < 1e-6
    assert np.max(np.abs(a.ps["Density"] - b.ps["Density"]) / a.ps["Density"]) < 1e-5
    # neighbour counts: the lattice puts many pairs exactly at q = 2 (2h = 3 dx), whose inclusion
    # follows the last bit of the positions; the total stays within a percent
    na, nb = int(a.ps["nCount"].sum()), int(b.ps["nCount"].sum())
    assert abs(na - nb) <= 0.01 * na
