"""Checkpoint / resume of a host particle system, in the reference's raw-writer files.

The reference saves `raw/int_properties` and `raw/float_properties` (the alive rows of the
property matrices) and `appendix/*` (TMSTEP, TimeValue, TimeStamp, WriteStep) to one JLD2 file per
output step (src/DataIO/Writer/RawWriter.jl:11-60), and `DataIO.load!` reads them back before a
restart (main.jl:150-156).  `save` writes that file (epp.jld2: the HDF5 layout written directly,
uncompressed) under the raw writer's names and naming scheme; a path ending in `.npz` gets the
same datasets in a NumPy archive instead.  `load` reads either.
"""
import os
import time

import numpy as np

from . import jld2


def appendix(step=0, time_value=0.0, write_step=0):
    """The reference's appendix dictionary (RawWriter.jl:19-21)."""
    return {"TMSTEP": int(step), "TimeValue": float(time_value), "TimeStamp": "", "WriteStep": int(write_step)}


def file_name(path, step, file_name="result", connect="_", digits=4, suffix=".jld2"):
    """Same naming as the raw writer (RawWriter.jl:23-28): path/result_0001.jld2."""
    return os.path.join(path, "%s%s%s%s" % (file_name, connect, str(step).zfill(digits), suffix))


def save(ps, path, app=None):
    """Alive rows of the int and float property matrices plus the appendix."""
    n = ps.n_particles
    mask = ps.is_alive[:n] == 1
    app = dict(app or appendix())
    app["TimeStamp"] = time.strftime("%Y_%m_%d_%H_%M_%S")
    raw = {"int_properties": np.ascontiguousarray(ps.int_properties[:n][mask]),
           "float_properties": np.ascontiguousarray(ps.float_properties[:n][mask])}
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    if not path.endswith(".npz"):   # the appendix first, as saveAppendix runs before the matrices
        return jld2.write(path, {"appendix": app, "raw": raw})
    arrays = {"raw/%s" % k: v for k, v in raw.items()}
    for k, v in app.items():
        arrays["appendix/%s" % k] = np.asarray(v)
    with open(path, "wb") as f:
        np.savez(f, **arrays)
    return path


def load(ps, path):
    """Restore the alive rows into `ps` (rows 0..m-1 alive, the rest dead, cells to be recomputed
    by the next search) and return the appendix."""
    with open(path, "rb") as f:
        npz = f.read(4) == b"PK\x03\x04"
    if npz:
        with np.load(path, allow_pickle=False) as z:
            ip = z["raw/int_properties"]
            fp = z["raw/float_properties"]
            app = {k.split("/", 1)[1]: z[k].item() for k in z.files if k.startswith("appendix/")}
    else:
        f = jld2.read(path)
        ip, fp, app = f["raw"]["int_properties"], f["raw"]["float_properties"], dict(f["appendix"])
    m = ip.shape[0]
    if m > ps.n_capacity or ip.shape[1] != ps.int_properties.shape[1] or fp.shape[1] != ps.float_properties.shape[1]:
        raise ValueError("checkpoint of %d rows x (%d, %d) columns does not fit this particle system" %
                         (m, ip.shape[1], fp.shape[1]))
    ps.int_properties[:] = 0
    ps.float_properties[:] = 0
    ps.int_properties[:m] = ip
    ps.float_properties[:m] = fp
    ps.is_alive[:] = 0
    ps.is_alive[:m] = 1
    ps.cell_index[:] = 0
    ps.set_n_particles(m)
    return app


def prepare_restart(ps, rate="dDensity"):
    """Clear the saved density rate before the restart's first search!: the search action adds
    the continuity rate to dDensity (Continuity.jl:23-47 accumulates; sContinuity! clears it only
    after use), so a rate saved after a search would otherwise be counted twice."""
    ps[rate] = np.zeros(ps.n_particles, np.float32)
