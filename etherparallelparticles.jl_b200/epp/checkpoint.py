"""Checkpoint / resume of a host particle system, with the datasets of the reference's raw writer.

The reference saves `raw/int_properties` and `raw/float_properties` (the alive rows of the
property matrices) and `appendix/*` (TMSTEP, TimeValue, TimeStamp, WriteStep) to one JLD2 file per
output step (src/DataIO/Writer/RawWriter.jl:11-60), and `DataIO.load!` reads them back before a
restart (main.jl:150-156).  JLD2 is an HDF5 container and no HDF5 library is available here, so
the same datasets go into a NumPy .npz archive under the same names; a Julia driver keeps using its
own writer on the matrices `epp_download` returns in the reference layout.
"""
import os
import time

import numpy as np


def appendix(step=0, time_value=0.0, write_step=0):
    """The reference's appendix dictionary (RawWriter.jl:19-21)."""
    return {"TMSTEP": int(step), "TimeValue": float(time_value), "TimeStamp": "", "WriteStep": int(write_step)}


def file_name(path, step, file_name="result", connect="_", digits=4, suffix=".npz"):
    """Same naming as the raw writer (RawWriter.jl:23-28): path/result_0001.npz."""
    return os.path.join(path, "%s%s%s%s" % (file_name, connect, str(step).zfill(digits), suffix))


def save(ps, path, app=None):
    """Alive rows of the int and float property matrices plus the appendix."""
    n = ps.n_particles
    mask = ps.is_alive[:n] == 1
    app = dict(app or appendix())
    app["TimeStamp"] = time.strftime("%Y_%m_%d_%H_%M_%S")
    arrays = {"raw/int_properties": np.ascontiguousarray(ps.int_properties[:n][mask]),
              "raw/float_properties": np.ascontiguousarray(ps.float_properties[:n][mask])}
    for k, v in app.items():
        arrays["appendix/%s" % k] = np.asarray(v)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        np.savez(f, **arrays)
    return path


def load(ps, path):
    """Restore the alive rows into `ps` (rows 0..m-1 alive, the rest dead, cells to be recomputed
    by the next search) and return the appendix."""
    with np.load(path, allow_pickle=False) as z:
        ip = z["raw/int_properties"]
        fp = z["raw/float_properties"]
        app = {k.split("/", 1)[1]: z[k].item() for k in z.files if k.startswith("appendix/")}
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
