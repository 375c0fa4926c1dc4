"""ctypes binding of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: it restates the reference on the CPU and checks the CUDA
path.  It is built by `make -C oracle` (or __graft_entry__.build()).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from epp import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

ORC_FIELD_POSITION = 0
ORC_FIELD_VELOCITY = 1
ORC_FIELD_DVELOCITY = 2
ORC_FIELD_DENSITY = 3
ORC_FIELD_DDENSITY = 4
ORC_FIELD_PRESSURE = 5
ORC_FIELD_VOLUME = 6
ORC_FIELD_MASS = 7
ORC_FIELD_ACCEL = 8
ORC_FIELD_NCOUNT = 9
ORC_FIELD_ACCEL_ABS = 10
ORC_FIELD_DDENSITY_ABS = 11

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    lib = C.CDLL(ORACLE_SO)
    P = C.POINTER
    i32p, f32p, f64p = P(C.c_int32), P(C.c_float), P(C.c_double)
    lib.orc_domain_info.argtypes = [P(abi.epp_domain), C.c_int32, i32p, f64p, f64p]
    lib.orc_cell_of.argtypes = [P(abi.epp_domain), C.c_int32, f32p, i32p, i32p, i32p]
    lib.orc_neighbour_cell_table.argtypes = [P(abi.epp_domain), i32p, i32p]
    lib.orc_kernel.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, f64p, f64p]
    lib.orc_kernel.restype = C.c_int32
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_int32, P(abi.epp_config)]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_set_threads.argtypes = [C.c_int32]
    lib.orc_set_deterministic.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_upload.argtypes = [C.c_void_p, C.c_int32, i32p, i32p, i32p, C.c_int64, f32p,
                               C.c_int64, P(abi.epp_column_map)]
    lib.orc_download.argtypes = [C.c_void_p, i32p, i32p, i32p, C.c_int64, f32p, C.c_int64,
                                 P(abi.epp_column_map)]
    lib.orc_get_field.argtypes = [C.c_void_p, C.c_int32, C.c_int32, f64p]
    lib.orc_set_field.argtypes = [C.c_void_p, C.c_int32, C.c_int32, f64p]
    lib.orc_search.argtypes = [C.c_void_p, C.c_int32, C.c_int32, P(abi.epp_physics), C.c_int32]
    lib.orc_interaction.argtypes = [C.c_void_p, C.c_int32, P(abi.epp_physics)]
    lib.orc_selfaction.argtypes = [C.c_void_p, C.c_int32, P(abi.epp_physics)]
    lib.orc_step.argtypes = [C.c_void_p, C.c_int32, P(abi.epp_physics)]
    lib.orc_integrals.argtypes = [C.c_void_p, P(abi.epp_physics), P(abi.epp_integrals)]
    lib.orc_cell_stats.argtypes = [C.c_void_p, i32p, i32p, i32p, i32p]
    lib.orc_step_dt.argtypes = [C.c_void_p, P(abi.epp_physics), f64p, f64p]
    lib.orc_status.restype = C.c_uint32
    lib.orc_status.argtypes = [C.c_void_p]
    _lib = lib
    return lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Oracle:
    """One oracle system (reference layout) at precision 32 or 64."""

    def __init__(self, config, precision=32):
        self.lib = load()
        self.config = config
        self.h = self.lib.orc_create(precision, C.byref(config))
        if not self.h:
            raise RuntimeError("orc_create failed")
        self.precision = precision

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def _ck(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s -> %s" % (what, abi.STATUS_NAMES.get(rc, rc)))

    def upload(self, n, is_alive, cell_index, ip, fp, cmap):
        self._ck(self.lib.orc_upload(self.h, n, _p(is_alive, C.c_int32), _p(cell_index, C.c_int32),
                                     _p(ip, C.c_int32), ip.shape[0], _p(fp, C.c_float), fp.shape[0],
                                     C.byref(cmap)), "orc_upload")

    def download(self, is_alive, cell_index, ip, fp, cmap):
        self._ck(self.lib.orc_download(self.h, _p(is_alive, C.c_int32), _p(cell_index, C.c_int32),
                                       _p(ip, C.c_int32), ip.shape[0] if ip is not None else 0,
                                       _p(fp, C.c_float), fp.shape[0] if fp is not None else 0,
                                       C.byref(cmap)), "orc_download")

    def field(self, field, k=0, n=None):
        n = n if n is not None else self.config.n_capacity
        out = np.zeros(self.config.n_capacity, dtype=np.float64)
        self._ck(self.lib.orc_get_field(self.h, field, k, _p(out, C.c_double)), "orc_get_field")
        return out[:n]

    def set_field(self, field, values, k=0):
        v = np.zeros(self.config.n_capacity, dtype=np.float64)
        v[: len(values)] = values
        self._ck(self.lib.orc_set_field(self.h, field, k, _p(v, C.c_double)), "orc_set_field")

    def search(self, criterion, action, phys=None, flags=0):
        self._ck(self.lib.orc_search(self.h, criterion, action,
                                     C.byref(phys) if phys is not None else None, flags), "orc_search")

    def interaction(self, action, phys=None):
        self._ck(self.lib.orc_interaction(self.h, action,
                                          C.byref(phys) if phys is not None else None), "orc_interaction")

    def selfaction(self, action, phys=None):
        self._ck(self.lib.orc_selfaction(self.h, action,
                                         C.byref(phys) if phys is not None else None), "orc_selfaction")

    def step(self, n, phys):
        self._ck(self.lib.orc_step(self.h, n, C.byref(phys)), "orc_step")

    def integrals(self, phys):
        out = abi.epp_integrals()
        self._ck(self.lib.orc_integrals(self.h, C.byref(phys), C.byref(out)), "orc_integrals")
        return out.as_dict()

    def cell_stats(self, n_alive):
        nc = C.c_int32(0)
        self._ck(self.lib.orc_cell_stats(self.h, None, None, None, C.byref(nc)), "orc_cell_stats")
        counts = np.zeros(nc.value, np.int32)
        offsets = np.zeros(nc.value + 1, np.int32)
        ids = np.zeros(max(n_alive, 1), np.int32)
        self._ck(self.lib.orc_cell_stats(self.h, _p(counts, C.c_int32), _p(offsets, C.c_int32),
                                         _p(ids, C.c_int32), C.byref(nc)), "orc_cell_stats")
        return counts, offsets, ids[:n_alive]

    def step_dt(self, phys):
        """(dt of the next step, simulated time since upload)."""
        dt, t = C.c_double(0), C.c_double(0)
        self._ck(self.lib.orc_step_dt(self.h, C.byref(phys), C.byref(dt), C.byref(t)), "orc_step_dt")
        return dt.value, t.value

    def status(self):
        return self.lib.orc_status(self.h)


def set_threads(n):
    load().orc_set_threads(n)


def kernel(kind, dim, r, hinv):
    """(W, dW/dr) of the oracle's kernel `kind` (FP64)."""
    lib = load()
    w, dw = C.c_double(0), C.c_double(0)
    rc = lib.orc_kernel(kind, dim, r, hinv, C.byref(w), C.byref(dw))
    if rc:
        raise RuntimeError("orc_kernel %d" % rc)
    return w.value, dw.value
