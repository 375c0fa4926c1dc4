"""ctypes mirror of include/epp.h (the C ABI of libepp.so).

Every struct and constant here has the same name, field order and meaning as in the header;
the header cites the reference interface each entry point replaces.
"""
import ctypes as C

EPP_ABI_VERSION = 4
EPP_TUNING_LISTS = 64   # epp_set_tuning: family 0 with the lockstep list search + continuity pass (2D)
EPP_MAX_TAGS = 16

# epp_status
EPP_OK = 0
EPP_ERR_INVALID_ARGUMENT = 1
EPP_ERR_CUDA = 2
EPP_ERR_OUT_OF_MEMORY = 3
EPP_ERR_UNSUPPORTED_ACTION = 4
EPP_ERR_UNSUPPORTED_CRITERION = 5
EPP_ERR_STATE = 6
EPP_ERR_DEVICE_STATUS = 7
EPP_ERR_BUDGET = 8
EPP_ERR_NO_DEVICE = 9
EPP_ERR_CAPACITY = 10

STATUS_NAMES = {
    EPP_OK: "EPP_OK",
    EPP_ERR_INVALID_ARGUMENT: "EPP_ERR_INVALID_ARGUMENT",
    EPP_ERR_CUDA: "EPP_ERR_CUDA",
    EPP_ERR_OUT_OF_MEMORY: "EPP_ERR_OUT_OF_MEMORY",
    EPP_ERR_UNSUPPORTED_ACTION: "EPP_ERR_UNSUPPORTED_ACTION",
    EPP_ERR_UNSUPPORTED_CRITERION: "EPP_ERR_UNSUPPORTED_CRITERION",
    EPP_ERR_STATE: "EPP_ERR_STATE",
    EPP_ERR_DEVICE_STATUS: "EPP_ERR_DEVICE_STATUS",
    EPP_ERR_BUDGET: "EPP_ERR_BUDGET",
    EPP_ERR_NO_DEVICE: "EPP_ERR_NO_DEVICE",
    EPP_ERR_CAPACITY: "EPP_ERR_CAPACITY",
}

# device status bits
EPP_STATUS_KILLED = 1 << 0
EPP_STATUS_NEIGHBOUR_OVERFLOW = 1 << 1
EPP_STATUS_CELL_OVERFLOW = 1 << 2
EPP_STATUS_NONFINITE = 1 << 3
EPP_STATUS_SPIN_TIMEOUT = 1 << 4
EPP_STATUS_BAD_TAG = 1 << 5
EPP_STATUS_QUEUE = 1 << 6

EPP_CRITERION_DEFAULT = 0
EPP_CRITERION_SYMMETRY = 1

EPP_ACTION_NONE = 0
EPP_ACTION_DAMBREAK_CONTINUITY = 1
EPP_ACTION_DAMBREAK_DENSITY = 2
EPP_ACTION_DAMBREAK_MOMENTUM = 3
EPP_ACTION_DAMBREAK_INTEGRATE = 4
EPP_ACTION_ZERO_DVELOCITY = 5
EPP_ACTION_COUNT_NEIGHBOURS = 6
EPP_ACTION_KERNEL_FILTER = 7
EPP_ACTION_KERNEL_FILTER_SELF = 8
EPP_ACTION_EXTRAPOLATE_PRESSURE = 9
EPP_ACTION_EXTRAPOLATE_PRESSURE_SELF = 10

EPP_SEARCH_EMIT_LIST = 1

EPP_INTEGRALS_SLOTS = 4
EPP_PROFILE_STAGES = 6   # momentum+integrate+bin, scan, scatter, rank+gather, search, continuity

EPP_VISCOSITY_REFERENCE = 0
EPP_VISCOSITY_MONAGHAN = 1
EPP_VISCOSITY_CLASSIC = 2

EPP_KERNEL_WENDLAND_C2 = 0
EPP_KERNEL_CUBIC_SPLINE = 1
EPP_KERNEL_GAUSSIAN = 2
EPP_KERNEL_WENDLAND_C4 = 3

EPP_EOS_TAIT = 0
EPP_EOS_LINEAR = 1

EPP_MOTION_SYMPLECTIC = 0
EPP_MOTION_ACCELERATE_MOVE = 1

EPP_PRESSURE_DEFAULT = 0
EPP_PRESSURE_CLASSIC = 1
EPP_PRESSURE_BALANCED = 2
EPP_PRESSURE_DENSITY_WEIGHTED = 3

EPP_WALL_PRESSURE_EOS = 0
EPP_WALL_PRESSURE_EXTRAPOLATE = 1


class epp_domain(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("gap", C.c_float),
        ("first", C.c_float * 3),
        ("last", C.c_float * 3),
    ]


class epp_physics(C.Structure):
    _fields_ = [
        ("dt", C.c_float),
        ("rho0", C.c_float),
        ("c0", C.c_float),
        ("p0", C.c_float),
        ("gamma", C.c_int32),
        ("gravity", C.c_float * 3),
        ("alpha", C.c_float),
        ("beta", C.c_float),
        ("viscosity", C.c_int32),
        ("fluid_tag", C.c_int32),
        ("wall_tag", C.c_int32),
        ("kahan", C.c_int32),
        ("kernel", C.c_int32),
        ("eos", C.c_int32),
        ("mu", C.c_float),
        ("motion", C.c_int32),
        ("filter_interval", C.c_int32),
        ("pressure_ff", C.c_int32),
        ("pressure_fw", C.c_int32),
        ("tensile", C.c_int32),
        ("wall_pressure", C.c_int32),
        ("cfl", C.c_float),
    ]


class epp_config(C.Structure):
    _fields_ = [
        ("domain", epp_domain),
        ("n_capacity", C.c_int32),
        ("max_neighbour_number", C.c_int32),
        ("max_cell_particles", C.c_int32),
        ("n_tags", C.c_int32),
        ("adjacency", C.c_int32 * (EPP_MAX_TAGS * EPP_MAX_TAGS)),
        ("device", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("n_instances", C.c_int32),
    ]


_COLUMN_FIELDS = [
    "tag", "is_movable", "n_count", "n_index",
    "position", "velocity", "dvelocity", "mass", "volume", "density", "ddensity", "pressure",
    "gap", "h", "n_rvec", "n_r", "n_w", "n_dw", "n_hinv", "instance",
]


class epp_column_map(C.Structure):
    _fields_ = [(f, C.c_int32) for f in _COLUMN_FIELDS]

    @classmethod
    def empty(cls):
        m = cls()
        for f in _COLUMN_FIELDS:
            setattr(m, f, -1)
        return m


class epp_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("peak_resident_bytes", C.c_int64),
        ("max_concurrent", C.c_int32),
        ("waiting", C.c_int32),
        ("active", C.c_int32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class epp_integrals(C.Structure):
    _fields_ = [
        ("mass_total", C.c_double),
        ("mass_fluid", C.c_double),
        ("kinetic", C.c_double),
        ("potential", C.c_double),
        ("internal", C.c_double),
        ("max_speed", C.c_double),
        ("cfl_dt", C.c_double),
        ("n_alive", C.c_int64),
        ("n_pairs", C.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def make_domain(dim, gap, first, last):
    d = epp_domain()
    d.dim = dim
    d.gap = gap
    for a in range(3):
        d.first[a] = first[a] if a < len(first) else 0.0
        d.last[a] = last[a] if a < len(last) else 0.0
    return d


def make_physics(dt, rho0=1000.0, c0=62.64, p0=0.0, gamma=7, gravity=(0.0, -9.81, 0.0),
                 alpha=0.1, beta=0.1, viscosity=EPP_VISCOSITY_REFERENCE, fluid_tag=1,
                 wall_tag=2, kahan=1, kernel=EPP_KERNEL_WENDLAND_C2, eos=EPP_EOS_TAIT, mu=0.0,
                 motion=EPP_MOTION_SYMPLECTIC, filter_interval=0, pressure_ff=EPP_PRESSURE_DEFAULT,
                 pressure_fw=EPP_PRESSURE_DEFAULT, tensile=0, wall_pressure=EPP_WALL_PRESSURE_EOS, cfl=0.0):
    p = epp_physics()
    p.dt = dt
    p.rho0 = rho0
    p.c0 = c0
    p.p0 = p0
    p.gamma = gamma
    for a in range(3):
        p.gravity[a] = gravity[a] if a < len(gravity) else 0.0
    p.alpha = alpha
    p.beta = beta
    p.viscosity = viscosity
    p.fluid_tag = fluid_tag
    p.wall_tag = wall_tag
    p.kahan = kahan
    p.kernel = kernel
    p.eos = eos
    p.mu = mu
    p.motion = motion
    p.filter_interval = filter_interval
    p.pressure_ff = pressure_ff
    p.pressure_fw = pressure_fw
    p.tensile = tensile
    p.wall_pressure = wall_pressure
    p.cfl = cfl
    return p


def make_config(domain, n_capacity, adjacency, max_neighbour_number=50, max_cell_particles=0,
                device=0, hbm_budget_bytes=0, n_instances=1):
    c = epp_config()
    c.domain = domain
    c.n_capacity = n_capacity
    c.max_neighbour_number = max_neighbour_number
    c.max_cell_particles = max_cell_particles
    n_tags = len(adjacency)
    if n_tags < 1 or n_tags > EPP_MAX_TAGS:
        raise ValueError("adjacency must be 1..%d square" % EPP_MAX_TAGS)
    c.n_tags = n_tags
    for i in range(n_tags):
        if len(adjacency[i]) != n_tags:
            raise ValueError("adjacency must be square")
        for j in range(n_tags):
            c.adjacency[i * EPP_MAX_TAGS + j] = int(adjacency[i][j])
    c.device = device
    c.hbm_budget_bytes = hbm_budget_bytes
    c.n_instances = n_instances
    return c
