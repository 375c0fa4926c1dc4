"""ctypes binding of libepp.so (include/epp.h).

The library is built in-tree (csrc/Makefile) next to this file.  There is no CPU fallback:
loading fails loudly when the library is missing, and every entry point raises EppError on a
non-zero status.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("EPP_LIB") or os.path.join(HERE, "libepp.so")

EXPORTS = [
    "epp_abi_version", "epp_device_count", "epp_create", "epp_destroy", "epp_last_error",
    "epp_upload", "epp_download", "epp_search", "epp_interaction", "epp_selfaction", "epp_step",
    "epp_get_integrals", "epp_cell_stats", "epp_synchronize", "epp_last_step_timing",
    "epp_pairs_total", "epp_set_accel_output", "epp_get_accel", "epp_set_stream",
    "epp_profile_step", "epp_set_tuning", "epp_cell_sort_noalloc", "epp_noalloc_limits",
    "epp_set_instance_physics", "epp_get_instance_integrals", "epp_context_bytes", "epp_query",
    "epp_set_priority", "epp_set_block_threads", "epp_integrals_async", "epp_integrals_wait",
    "epp_server_create", "epp_server_destroy", "epp_server_submit", "epp_server_poll", "epp_server_drain",
    "epp_server_result", "epp_server_download", "epp_server_set_co_batch", "epp_neighbour_lists",
    "epp_step_dt",
]


def context_bytes(config):
    """Device bytes a context of this configuration allocates (epp_context_bytes)."""
    lib = load()
    b = C.c_int64(0)
    rc = lib.epp_context_bytes(C.byref(config), C.byref(b))
    if rc != abi.EPP_OK:
        raise EppError(rc, "epp_context_bytes")
    return b.value


class EppError(RuntimeError):
    def __init__(self, code, what, detail=""):
        self.code = code
        super().__init__("%s -> %s %s" % (what, abi.STATUS_NAMES.get(code, code), detail))


_lib = None


def load(path=LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libepp.so is not built (%s); run __graft_entry__.build() or make -C "
                          "etherparallelparticles.jl_b200/csrc" % path)
    lib = C.CDLL(path)
    P = C.POINTER
    i32p, f32p = P(C.c_int32), P(C.c_float)
    ctx = C.c_void_p
    lib.epp_abi_version.restype = C.c_int32
    lib.epp_device_count.argtypes = [i32p]
    lib.epp_create.argtypes = [P(abi.epp_config), P(C.c_void_p)]
    lib.epp_destroy.argtypes = [ctx]
    lib.epp_last_error.restype = C.c_char_p
    lib.epp_last_error.argtypes = [ctx]
    lib.epp_upload.argtypes = [ctx, C.c_int32, i32p, i32p, i32p, C.c_int64, f32p, C.c_int64,
                               P(abi.epp_column_map)]
    lib.epp_download.argtypes = [ctx, i32p, i32p, i32p, C.c_int64, f32p, C.c_int64,
                                 P(abi.epp_column_map)]
    lib.epp_search.argtypes = [ctx, C.c_int32, C.c_int32, P(abi.epp_physics), C.c_int32]
    lib.epp_interaction.argtypes = [ctx, C.c_int32, P(abi.epp_physics)]
    lib.epp_selfaction.argtypes = [ctx, C.c_int32, P(abi.epp_physics)]
    lib.epp_step.argtypes = [ctx, C.c_int32, P(abi.epp_physics)]
    lib.epp_get_integrals.argtypes = [ctx, P(abi.epp_physics), P(abi.epp_integrals)]
    lib.epp_integrals_async.argtypes = [ctx, P(abi.epp_physics), P(C.c_int64)]
    srv = C.c_void_p
    lib.epp_server_create.argtypes = [C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.c_int32, P(C.c_void_p)]
    lib.epp_server_destroy.argtypes = [srv]
    lib.epp_server_set_co_batch.argtypes = [srv, C.c_int32, C.c_int32]
    lib.epp_server_submit.argtypes = [srv, P(abi.epp_config), C.c_int32, i32p, i32p, i32p, C.c_int64, f32p,
                                      C.c_int64, P(abi.epp_column_map), P(abi.epp_physics), C.c_int32, C.c_int32,
                                      P(C.c_int64)]
    lib.epp_server_poll.argtypes = [srv, P(abi.epp_server_stats)]
    lib.epp_server_drain.argtypes = [srv, P(abi.epp_server_stats)]
    lib.epp_server_result.argtypes = [srv, C.c_int64, P(abi.epp_integrals), P(C.c_uint32), P(C.c_double),
                                      P(C.c_double)]
    lib.epp_server_download.argtypes = [srv, C.c_int64, i32p, i32p, i32p, C.c_int64, f32p, C.c_int64]
    lib.epp_integrals_wait.argtypes = [ctx, C.c_int64, P(abi.epp_integrals)]
    lib.epp_cell_stats.argtypes = [ctx, i32p, i32p, i32p, i32p]
    lib.epp_neighbour_lists.argtypes = [ctx, i32p, i32p, C.c_int64, C.c_int32]
    lib.epp_step_dt.argtypes = [ctx, P(abi.epp_physics), C.c_int32, f32p, P(C.c_double)]
    lib.epp_synchronize.argtypes = [ctx, P(C.c_uint32)]
    lib.epp_last_step_timing.argtypes = [ctx, f32p]
    lib.epp_pairs_total.argtypes = [ctx, P(C.c_int64)]
    lib.epp_set_accel_output.argtypes = [ctx, C.c_int32]
    lib.epp_get_accel.argtypes = [ctx, f32p, C.c_int32]
    lib.epp_set_stream.argtypes = [ctx, C.c_void_p]
    lib.epp_profile_step.argtypes = [ctx, P(abi.epp_physics), f32p]
    lib.epp_set_tuning.argtypes = [ctx, C.c_int32]
    lib.epp_cell_sort_noalloc.argtypes = [P(abi.epp_domain), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, i32p, C.c_void_p]
    lib.epp_noalloc_limits.argtypes = [i32p, i32p, P(C.c_int64)]
    lib.epp_set_instance_physics.argtypes = [ctx, C.c_int32, f32p, f32p]
    lib.epp_get_instance_integrals.argtypes = [ctx, P(abi.epp_physics), P(abi.epp_integrals), C.c_int32]
    lib.epp_context_bytes.argtypes = [P(abi.epp_config), P(C.c_int64)]
    lib.epp_query.argtypes = [ctx, i32p]
    lib.epp_set_priority.argtypes = [ctx, C.c_int32, i32p]
    lib.epp_set_block_threads.argtypes = [ctx, C.c_int32]
    for name in EXPORTS:
        if name not in ("epp_last_error", "epp_abi_version"):
            getattr(lib, name).restype = C.c_int32
    if lib.epp_abi_version() != abi.EPP_ABI_VERSION:
        raise ImportError("libepp ABI %d != %d" % (lib.epp_abi_version(), abi.EPP_ABI_VERSION))
    _lib = lib
    return lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Context:
    """One device context (epp_ctx) holding a particle system's state on a GPU."""

    def __init__(self, config):
        self.lib = load()
        self.config = config
        h = C.c_void_p()
        rc = self.lib.epp_create(C.byref(config), C.byref(h))
        if rc != abi.EPP_OK:
            raise EppError(rc, "epp_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.epp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != abi.EPP_OK:
            detail = self.lib.epp_last_error(self.h).decode() if self.h else ""
            raise EppError(rc, what, detail)

    def upload(self, n, is_alive, cell_index, int_props, float_props, cmap):
        self._ck(self.lib.epp_upload(self.h, n, _ptr(is_alive, C.c_int32), _ptr(cell_index, C.c_int32),
                                     _ptr(int_props, C.c_int32), int_props.shape[0],
                                     _ptr(float_props, C.c_float), float_props.shape[0], C.byref(cmap)),
                 "epp_upload")

    def download(self, is_alive, cell_index, int_props, float_props, cmap):
        self._ck(self.lib.epp_download(self.h, _ptr(is_alive, C.c_int32), _ptr(cell_index, C.c_int32),
                                       _ptr(int_props, C.c_int32),
                                       int_props.shape[0] if int_props is not None else 0,
                                       _ptr(float_props, C.c_float),
                                       float_props.shape[0] if float_props is not None else 0,
                                       C.byref(cmap)), "epp_download")

    def search(self, criterion, action, phys=None, flags=0):
        self._ck(self.lib.epp_search(self.h, criterion, action,
                                     C.byref(phys) if phys is not None else None, flags), "epp_search")

    def interaction(self, action, phys=None):
        self._ck(self.lib.epp_interaction(self.h, action, C.byref(phys) if phys is not None else None),
                 "epp_interaction")

    def selfaction(self, action, phys=None):
        self._ck(self.lib.epp_selfaction(self.h, action, C.byref(phys) if phys is not None else None),
                 "epp_selfaction")

    def step(self, n_steps, phys):
        self._ck(self.lib.epp_step(self.h, n_steps, C.byref(phys)), "epp_step")

    def integrals(self, phys):
        out = abi.epp_integrals()
        self._ck(self.lib.epp_get_integrals(self.h, C.byref(phys), C.byref(out)), "epp_get_integrals")
        return out.as_dict()

    def integrals_async(self, phys):
        """Enqueue the integrals of the current state; returns a ticket for integrals_wait."""
        t = C.c_int64(-1)
        self._ck(self.lib.epp_integrals_async(self.h, C.byref(phys), C.byref(t)), "epp_integrals_async")
        return t.value

    def integrals_wait(self, ticket):
        out = abi.epp_integrals()
        self._ck(self.lib.epp_integrals_wait(self.h, C.c_int64(ticket), C.byref(out)), "epp_integrals_wait")
        return out.as_dict()

    def cell_stats(self):
        import numpy as np
        nc = C.c_int32(0)
        self._ck(self.lib.epp_cell_stats(self.h, None, None, None, C.byref(nc)), "epp_cell_stats")
        counts = np.zeros(nc.value, np.int32)
        offsets = np.zeros(nc.value + 1, np.int32)
        self._ck(self.lib.epp_cell_stats(self.h, _ptr(counts, C.c_int32), _ptr(offsets, C.c_int32), None,
                                         C.byref(nc)), "epp_cell_stats")
        ids = np.zeros(max(int(offsets[-1]), 1), np.int32)
        self._ck(self.lib.epp_cell_stats(self.h, None, None, _ptr(ids, C.c_int32), C.byref(nc)),
                 "epp_cell_stats")
        return counts, offsets, ids[: int(offsets[-1])]

    def step_dt(self, phys, n=1):
        """(next_dt[n], sim_time[n]): the dt of the next step per instance and the simulated time
        advanced by epp_step since the last upload (epp_step_dt)."""
        import numpy as np
        dt = np.zeros(n, np.float32)
        t = np.zeros(n, np.float64)
        self._ck(self.lib.epp_step_dt(self.h, C.byref(phys), n, _ptr(dt, C.c_float), _ptr(t, C.c_double)),
                 "epp_step_dt")
        return dt, t

    def neighbour_lists(self, n, max_nb):
        """(counts[n], ids[n, max_nb]): nCount per caller row and the 1-based neighbour ids of the
        search pass's lists (epp_neighbour_lists), in list order; unused slots are 0."""
        import numpy as np
        counts = np.zeros(n, np.int32)
        ids = np.zeros((max_nb, max(n, 1)), np.int32)   # ids[k, row]: column-major with ld = n
        self._ck(self.lib.epp_neighbour_lists(self.h, _ptr(counts, C.c_int32), _ptr(ids, C.c_int32), max(n, 1),
                                              max_nb), "epp_neighbour_lists")
        return counts, ids[:, :n].T.copy()

    def synchronize(self, raise_on_status=True):
        st = C.c_uint32(0)
        rc = self.lib.epp_synchronize(self.h, C.byref(st))
        if rc == abi.EPP_ERR_DEVICE_STATUS and not raise_on_status:
            return st.value
        self._ck(rc, "epp_synchronize")
        return st.value

    def last_step_ms(self):
        v = C.c_float(0)
        self._ck(self.lib.epp_last_step_timing(self.h, C.byref(v)), "epp_last_step_timing")
        return v.value

    def pairs_total(self):
        v = C.c_int64(0)
        self._ck(self.lib.epp_pairs_total(self.h, C.byref(v)), "epp_pairs_total")
        return v.value

    def set_accel_output(self, enable):
        self._ck(self.lib.epp_set_accel_output(self.h, 1 if enable else 0), "epp_set_accel_output")

    def set_instance_physics(self, dt, c0):
        import numpy as np
        dt = np.ascontiguousarray(dt, dtype=np.float32)
        c0 = np.ascontiguousarray(c0, dtype=np.float32)
        self._ck(self.lib.epp_set_instance_physics(self.h, len(dt), _ptr(dt, C.c_float), _ptr(c0, C.c_float)),
                 "epp_set_instance_physics")

    def instance_integrals(self, phys, n):
        out = (abi.epp_integrals * n)()
        self._ck(self.lib.epp_get_instance_integrals(self.h, C.byref(phys), out, n), "epp_get_instance_integrals")
        return [o.as_dict() for o in out]

    def done(self):
        """True when all work queued on this context has finished (non-blocking)."""
        d = C.c_int32(0)
        self._ck(self.lib.epp_query(self.h, C.byref(d)), "epp_query")
        return bool(d.value)

    def set_priority(self, priority):
        """CUDA stream priority of the context's own stream (lower = first); returns the value used."""
        a = C.c_int32(0)
        self._ck(self.lib.epp_set_priority(self.h, priority, C.byref(a)), "epp_set_priority")
        return a.value

    def set_block_threads(self, threads):
        self._ck(self.lib.epp_set_block_threads(self.h, threads), "epp_set_block_threads")

    def set_tuning(self, lanes_per_particle):
        self._ck(self.lib.epp_set_tuning(self.h, lanes_per_particle), "epp_set_tuning")

    def set_stream(self, stream_handle):
        """Queue work on a caller-owned cudaStream_t (integer handle); None restores the own stream."""
        self._ck(self.lib.epp_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None),
                 "epp_set_stream")

    def profile_step(self, phys):
        """One step kernel by kernel; returns the EPP_PROFILE_STAGES stage times in ms."""
        out = (C.c_float * abi.EPP_PROFILE_STAGES)()
        self._ck(self.lib.epp_profile_step(self.h, C.byref(phys), out), "epp_profile_step")
        return list(out)

    def accel(self, n, dim):
        import numpy as np
        out = np.zeros(dim * n, np.float32)
        self._ck(self.lib.epp_get_accel(self.h, _ptr(out, C.c_float), n), "epp_get_accel")
        return out.reshape(dim, n).T.copy()


class NativeServer:
    """The native serving loop (epp_server_*): submit reference-layout states, poll or drain,
    read each request's integrals and (with keep_state) its final state."""

    def __init__(self, device=0, budget_bytes=120 * 10**9, max_active=256, chunk_steps=100, ahead=2,
                 co_batch=False, batch_max=256):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.epp_server_create(device, int(budget_bytes), max_active, chunk_steps, ahead, C.byref(h))
        if rc != abi.EPP_OK:
            raise EppError(rc, "epp_server_create")
        self.h = h
        if co_batch:
            self._ck(self.lib.epp_server_set_co_batch(self.h, 1, batch_max), "epp_server_set_co_batch")

    def close(self):
        if getattr(self, "h", None):
            self.lib.epp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        if rc != abi.EPP_OK:
            raise EppError(rc, what)

    def submit(self, config, ps, cmap, phys, steps, keep_state=False):
        """Queue the simulation held by particle system `ps` (copied now); returns its id."""
        rid = C.c_int64(-1)
        self._ck(self.lib.epp_server_submit(
            self.h, C.byref(config), ps.n_particles, _ptr(ps.is_alive, C.c_int32), _ptr(ps.cell_index, C.c_int32),
            _ptr(ps.int_properties, C.c_int32), ps.int_properties.shape[0], _ptr(ps.float_properties, C.c_float),
            ps.float_properties.shape[0], C.byref(cmap), C.byref(phys), steps, 1 if keep_state else 0,
            C.byref(rid)), "epp_server_submit")
        return rid.value

    def poll(self):
        st = abi.epp_server_stats()
        self._ck(self.lib.epp_server_poll(self.h, C.byref(st)), "epp_server_poll")
        return st.as_dict()

    def drain(self):
        st = abi.epp_server_stats()
        self._ck(self.lib.epp_server_drain(self.h, C.byref(st)), "epp_server_drain")
        return st.as_dict()

    def result(self, rid):
        out = abi.epp_integrals()
        status, a, d = C.c_uint32(0), C.c_double(0), C.c_double(0)
        self._ck(self.lib.epp_server_result(self.h, rid, C.byref(out), C.byref(status), C.byref(a), C.byref(d)),
                 "epp_server_result")
        return {"integrals": out.as_dict(), "status": status.value, "admit_s": a.value, "done_s": d.value}

    def download(self, rid, ps):
        """The final state of a keep_state request, into particle system `ps` (same layout)."""
        self._ck(self.lib.epp_server_download(
            self.h, rid, _ptr(ps.is_alive, C.c_int32), _ptr(ps.cell_index, C.c_int32),
            _ptr(ps.int_properties, C.c_int32), ps.int_properties.shape[0], _ptr(ps.float_properties, C.c_float),
            ps.float_properties.shape[0]), "epp_server_download")
