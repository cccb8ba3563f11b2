"""ctypes binding of libmmnb.so (include/mmnb.h).

The shared library is built in-tree by molmodel_b200/csrc/Makefile.  There is
no fallback: if it is missing, or no CUDA device is present when a potential is
created, the call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmmnb.so")

MMNB_OK = 0
MMNB_FP64 = 0
MMNB_MIXED = 1
MMNB_CUBIC = 1
MMNB_ORTHORHOMBIC = 2

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)
_vp = ctypes.c_void_p


class MmnbConfig(ctypes.Structure):
    """struct mmnb_config (include/mmnb.h)."""
    _fields_ = [
        ("precision", ctypes.c_int),
        ("bctype", ctypes.c_int),
        ("box", ctypes.c_double * 3),
        ("rspace_cutoff", ctypes.c_double),
        ("smoothing_width", ctypes.c_double),
        ("neighbor_list_width", ctypes.c_double),
        ("kspace_cutoff", ctypes.c_double),
        ("ewald_screening", ctypes.c_double),
        ("use_p3m", ctypes.c_int),
        ("p3m_grid_spacing", ctypes.c_double),
        ("p3m_assignment_order", ctypes.c_int),
        ("p3m_alias_sum_limit", ctypes.c_int),
        ("p3m_ik_differentiate", ctypes.c_int),
        ("include_lj_correction", ctypes.c_int),
        ("geometric_combining_for_sigma", ctypes.c_int),
        ("include_rspace", ctypes.c_int),
        ("include_kspace", ctypes.c_int),
        ("include_self", ctypes.c_int),
        ("elec_1_4_scale_factor", ctypes.c_double),
        ("lj_1_4_scale_factor", ctypes.c_double),
        ("rebuild_interval", ctypes.c_int),
        ("device", ctypes.c_int),
        ("p3m_grid_density", ctypes.c_double),
    ]


class MmnbEnergy(ctypes.Structure):
    _fields_ = [("elec", ctypes.c_double), ("lj", ctypes.c_double),
                ("lj_correction", ctypes.c_double), ("total", ctypes.c_double)]


# (name, restype, argtypes) for every entry point of include/mmnb.h
SIGNATURES = [
    ("mmnb_config_init", ctypes.c_int, [ctypes.POINTER(MmnbConfig)]),
    ("mmnb_create", ctypes.c_int, [ctypes.POINTER(MmnbConfig), ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                   ctypes.c_int, _ip, ctypes.POINTER(_vp)]),
    ("mmnb_set_params", ctypes.c_int, [_vp, _ip, _dp, _dp, _dp, _dp]),
    # untyped pointers: the per-step host call passes raw addresses (typed
    # pointer objects and byref() are accepted as well)
    ("mmnb_compute", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("mmnb_compute_device", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("mmnb_graph_capture", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("mmnb_graph_launch", ctypes.c_int, [_vp]),
    ("mmnb_scale", ctypes.c_int, [_vp, ctypes.c_double]),
    ("mmnb_set_stream", ctypes.c_int, [_vp, _vp]),
    ("mmnb_get_pairlist", ctypes.c_int, [_vp, _lp, _ip, ctypes.c_long]),
    ("mmnb_get_cells", ctypes.c_int, [_vp, _ip, _ip]),
    ("mmnb_get_counters", ctypes.c_int, [_vp, _lp, _lp]),
    ("mmnb_get_launches", ctypes.c_int, [_vp, _lp]),
    ("mmnb_check", ctypes.c_int, [_vp, _lp, _ip]),
    ("mmnb_get_settings", ctypes.c_int, [_vp, _dp, _dp, _dp, _ip]),
    ("mmnb_get_error_estimates", ctypes.c_int, [_vp, _dp, _dp]),
    ("mmnb_set_timing", ctypes.c_int, [_vp, ctypes.c_int]),
    ("mmnb_get_timing", ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    ("mmnb_destroy", ctypes.c_int, [_vp]),
    ("mmnb_last_error", ctypes.c_char_p, [_vp]),
    ("mmnb_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("mmnb_chebyshev_table", ctypes.c_int, [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]),
    ("mmnb_p3m_mesh_size", ctypes.c_int, [ctypes.c_double, ctypes.c_double]),
    ("mmnb_kspace_field_noalloc", ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, _dp, ctypes.c_double,
                                                 ctypes.c_double, _vp, _vp, _vp]),
    ("mmnb_measure_fp32_peak", ctypes.c_int, [ctypes.c_int, _dp]),
    ("mmnb_autotune", ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    ("mmnb_get_tuning", ctypes.c_int, [_vp, _ip]),
    ("mmnb_set_tuning", ctypes.c_int, [_vp, _ip]),
    ("mmnb_backward", ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("mmnb_forward", ctypes.c_int, [_vp, _dp, _dp, _dp, ctypes.POINTER(MmnbEnergy)]),
    ("mmnb_site_gradients", ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("mmnb_phi_at_points", ctypes.c_int, [_vp, _dp, ctypes.c_int, _dp, _dp]),
    ("mmnb_virial", ctypes.c_int, [_vp, _dp, ctypes.c_int, _ip, _dp, _dp, _dp, ctypes.POINTER(MmnbEnergy), _dp]),
    ("mmnb_md_create", ctypes.c_int, [_vp, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.POINTER(_vp)]),
    ("mmnb_md_set_state", ctypes.c_int, [_vp, _dp, _dp]),
    ("mmnb_md_run", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("mmnb_md_get_state", ctypes.c_int, [_vp, _dp, _dp]),
    ("mmnb_md_last_error", ctypes.c_char_p, [_vp]),
    ("mmnb_md_destroy", ctypes.c_int, [_vp]),
    ("mmnb_md_scale_velocities", ctypes.c_int, [_vp, ctypes.c_double]),
    ("mmnb_md_batch_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)]),
    ("mmnb_md_batch_run", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_dp)]),
    ("mmnb_md_batch_last_error", ctypes.c_char_p, [_vp]),
    ("mmnb_md_batch_destroy", ctypes.c_int, [_vp]),
]

_lib = None


def load():
    """Load libmmnb.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C molmodel_b200/csrc` "
                "(or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class MmnbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def check(status, handle=None):
    if status != MMNB_OK:
        lib = load()
        msg = lib.mmnb_last_error(handle).decode()
        raise MmnbError(status, msg or lib.mmnb_status_string(status).decode())
