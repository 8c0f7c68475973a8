"""ctypes binding of libmpdx.so (the C ABI declared in include/mpdx.h).

The shared library is built in-tree by __graft_entry__.build() (or `make -C
libmpdataxx_b200/csrc`).  There is no fallback: if the library is missing the
import of this module's `lib()` raises, and on a machine without a CUDA device
every solver call fails with the CUDA runtime's message.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# MPDX_LIBRARY=debug loads the bounds-checked, NaN-poisoned build (libmpdx_debug.so)
SO_PATH = os.path.join(HERE, "libmpdx_debug.so" if os.environ.get("MPDX_LIBRARY") == "debug" else "libmpdx.so")

MPDX_OK, MPDX_E_GRID, MPDX_E_DIVERGENT, MPDX_E_PRS_STUCK, MPDX_E_UNSUPPORTED, MPDX_E_CUDA, MPDX_E_TIMEOUT, MPDX_E_ARG = range(8)
BC = {"cyclic": 0, "open": 1, "rigid": 2, "gndsky": 3}
SOLVER_MPDATA, SOLVER_BOUSSINESQ = 0, 1
PRS_CR, PRS_GCRK = 0, 1
PRECOND_IDENTITY, PRECOND_LEARNED = 0, 1
PATH_AUTO, PATH_GENERAL, PATH_FUSED = 0, 1, 2
FIELD_ADVECTEE, FIELD_ADVECTOR, FIELD_SCLR_ARRAY, FIELD_PRESSURE, FIELD_G = 0, 1, 2, 3, 4
SCLR_THT_E = 0
SCLR_THT_ABS = 1
SCLR_HFLUX_FRC = 2
SCLR_VAB_COEFF = 3
SCLR_VAB_RELAX = 4  # + d
VAB_NONE, VAB_EXPL, VAB_IMPL = 0, 1, 2

# every entry point declared in include/mpdx.h
EXPORTS = ["mpdx_config_default", "mpdx_create", "mpdx_set_field", "mpdx_get_field", "mpdx_set_field_device",
           "mpdx_get_field_device", "mpdx_set_field_async", "mpdx_get_field_async", "mpdx_advance", "mpdx_sync", "mpdx_stats", "mpdx_stream", "mpdx_fused3d_bulk_copies", "mpdx_fused3d_planes_per_cta",
           "mpdx_fused3d_tuning", "mpdx_last_error",
           "mpdx_create_error", "mpdx_destroy", "mpdx_field_stats_noalloc", "mpdx_batch_create", "mpdx_batch_advance",
           "mpdx_batch_get_info", "mpdx_batch_sync", "mpdx_batch_last_error", "mpdx_batch_destroy",
           "mpdx_pcnet_create", "mpdx_pcnet_create_error", "mpdx_pcnet_num_params", "mpdx_pcnet_set_params",
           "mpdx_pcnet_get_params", "mpdx_pcnet_forward", "mpdx_pcnet_backward", "mpdx_pcnet_train_step",
           "mpdx_pcnet_last_error", "mpdx_pcnet_destroy", "mpdx_precond_record", "mpdx_precond_train",
           "mpdx_precond_enable", "mpdx_precond_directions", "mpdx_precond_set_directions", "mpdx_precond_pairs", "mpdx_precond_num_params", "mpdx_precond_get_params",
           "mpdx_precond_set_params", "mpdx_precond_loss_grad"]
BATCH_PERSISTENT, BATCH_PER_PROBLEM = 0, 1


class Config(ctypes.Structure):
    _fields_ = [("solver", ctypes.c_int), ("n_dims", ctypes.c_int), ("n_eqns", ctypes.c_int),
                ("grid", ctypes.c_int * 3), ("opts", ctypes.c_uint64), ("n_iters", ctypes.c_int),
                ("dtype", ctypes.c_int), ("bcs", ctypes.c_int * 6), ("dt", ctypes.c_double),
                ("di", ctypes.c_double), ("dj", ctypes.c_double), ("dk", ctypes.c_double),
                ("max_abs_div_eps", ctypes.c_double), ("path", ctypes.c_int), ("prs_scheme", ctypes.c_int),
                ("prs_k_iters", ctypes.c_int), ("prs_tol", ctypes.c_double), ("g", ctypes.c_double),
                ("tht_ref", ctypes.c_double), ("ix_u", ctypes.c_int), ("ix_v", ctypes.c_int),
                ("ix_w", ctypes.c_int), ("ix_tht", ctypes.c_int), ("precond", ctypes.c_int),
                ("prs_fp64", ctypes.c_int), ("upwind_filter_freq", ctypes.c_int),
                ("impl_tht", ctypes.c_int), ("vip_vab", ctypes.c_int), ("sptl_intrp", ctypes.c_int)]


class StepStats(ctypes.Structure):
    _fields_ = [("timestep", ctypes.c_int64), ("time", ctypes.c_double), ("mass", ctypes.c_double),
                ("min", ctypes.c_double), ("max", ctypes.c_double), ("gcr_iters", ctypes.c_int64),
                ("gcr_iters_total", ctypes.c_int64), ("gcr_residual", ctypes.c_double), ("path", ctypes.c_int),
                ("gcr_ms", ctypes.c_double), ("gcr_fallback", ctypes.c_int)]


class Tuning3D(ctypes.Structure):
    """mpdx_tuning3d: the fused 3D kernel's chunk-length tuner of one handle."""
    _fields_ = [("chosen", ctypes.c_int), ("n_candidates", ctypes.c_int), ("lx", ctypes.c_int * 8),
                ("ms", ctypes.c_float * 8)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("n_problems", ctypes.c_int), ("cells", ctypes.c_int64), ("mode", ctypes.c_int),
                ("tile_nt", ctypes.c_int), ("tile_lx", ctypes.c_int), ("grid", ctypes.c_int),
                ("n_candidates", ctypes.c_int), ("tune_ms", ctypes.c_double * 8)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO_PATH):
        raise ImportError(f"{SO_PATH} is not built; run __graft_entry__.build() (or make -C libmpdataxx_b200/csrc)")
    L = ctypes.CDLL(SO_PATH)
    vp, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
    L.mpdx_config_default.argtypes = [ctypes.POINTER(Config)]
    L.mpdx_config_default.restype = None
    L.mpdx_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.mpdx_create.restype = ctypes.c_int
    L.mpdx_create_error.argtypes = []
    L.mpdx_create_error.restype = ctypes.c_char_p
    for f in ("mpdx_set_field", "mpdx_get_field"):
        getattr(L, f).argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, i64p]
        getattr(L, f).restype = ctypes.c_int
    for f in ("mpdx_set_field_device", "mpdx_get_field_device", "mpdx_set_field_async", "mpdx_get_field_async"):
        getattr(L, f).argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        getattr(L, f).restype = ctypes.c_int
    L.mpdx_advance.argtypes = [vp, ctypes.c_int64]
    L.mpdx_advance.restype = ctypes.c_int
    L.mpdx_sync.argtypes = [vp]
    L.mpdx_sync.restype = ctypes.c_int
    L.mpdx_stats.argtypes = [vp, ctypes.POINTER(StepStats)]
    L.mpdx_stats.restype = ctypes.c_int
    L.mpdx_stream.argtypes = [vp]
    L.mpdx_stream.restype = vp
    L.mpdx_fused3d_bulk_copies.argtypes = [ctypes.c_int]
    L.mpdx_fused3d_bulk_copies.restype = ctypes.c_int
    L.mpdx_fused3d_planes_per_cta.argtypes = [ctypes.c_int]
    L.mpdx_fused3d_planes_per_cta.restype = ctypes.c_int
    L.mpdx_fused3d_tuning.argtypes = [vp, ctypes.POINTER(Tuning3D)]
    L.mpdx_fused3d_tuning.restype = ctypes.c_int
    L.mpdx_last_error.argtypes = [vp]
    L.mpdx_last_error.restype = ctypes.c_char_p
    L.mpdx_destroy.argtypes = [vp]
    L.mpdx_destroy.restype = None
    L.mpdx_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.mpdx_batch_create.restype = ctypes.c_int
    L.mpdx_batch_advance.argtypes = [vp, ctypes.c_int64]
    L.mpdx_batch_advance.restype = ctypes.c_int
    L.mpdx_batch_get_info.argtypes = [vp, ctypes.POINTER(BatchInfo)]
    L.mpdx_batch_get_info.restype = ctypes.c_int
    L.mpdx_batch_sync.argtypes = [vp]
    L.mpdx_batch_sync.restype = ctypes.c_int
    L.mpdx_batch_last_error.argtypes = [vp]
    L.mpdx_batch_last_error.restype = ctypes.c_char_p
    L.mpdx_batch_destroy.argtypes = [vp]
    L.mpdx_batch_destroy.restype = None
    ip, fp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
    L.mpdx_pcnet_create.argtypes = [ctypes.c_int, ip, ip, ip, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.mpdx_pcnet_create.restype = ctypes.c_int
    L.mpdx_pcnet_create_error.argtypes = []
    L.mpdx_pcnet_create_error.restype = ctypes.c_char_p
    L.mpdx_pcnet_num_params.argtypes = [vp]
    L.mpdx_pcnet_num_params.restype = ctypes.c_int64
    for f in ("mpdx_pcnet_set_params", "mpdx_pcnet_get_params"):
        getattr(L, f).argtypes = [vp, fp]
        getattr(L, f).restype = ctypes.c_int
    L.mpdx_pcnet_forward.argtypes = [vp, fp, fp]
    L.mpdx_pcnet_forward.restype = ctypes.c_int
    L.mpdx_pcnet_backward.argtypes = [vp, fp, fp, fp]
    L.mpdx_pcnet_backward.restype = ctypes.c_int
    L.mpdx_pcnet_train_step.argtypes = [vp, fp, fp, ctypes.c_float, ctypes.POINTER(ctypes.c_double)]
    L.mpdx_pcnet_train_step.restype = ctypes.c_int
    L.mpdx_pcnet_last_error.argtypes = [vp]
    L.mpdx_pcnet_last_error.restype = ctypes.c_char_p
    L.mpdx_pcnet_destroy.argtypes = [vp]
    L.mpdx_pcnet_destroy.restype = None
    L.mpdx_precond_record.argtypes = [vp, ctypes.c_int64]
    L.mpdx_precond_record.restype = ctypes.c_int
    L.mpdx_precond_train.argtypes = [vp, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    L.mpdx_precond_train.restype = ctypes.c_int
    L.mpdx_precond_enable.argtypes = [vp, ctypes.c_int]
    L.mpdx_precond_enable.restype = ctypes.c_int
    L.mpdx_precond_set_directions.argtypes = [vp, ctypes.c_int64]
    L.mpdx_precond_set_directions.restype = ctypes.c_int
    L.mpdx_precond_directions.argtypes = [vp]
    L.mpdx_precond_directions.restype = ctypes.c_int64
    L.mpdx_precond_pairs.argtypes = [vp]
    L.mpdx_precond_pairs.restype = ctypes.c_int64
    L.mpdx_precond_num_params.argtypes = [vp]
    L.mpdx_precond_num_params.restype = ctypes.c_int64
    L.mpdx_precond_get_params.argtypes = [vp, fp]
    L.mpdx_precond_get_params.restype = ctypes.c_int
    L.mpdx_precond_set_params.argtypes = [vp, fp]
    L.mpdx_precond_set_params.restype = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    L.mpdx_precond_loss_grad.argtypes = [vp, dp, dp, ctypes.c_double, dp, fp]
    L.mpdx_precond_loss_grad.restype = ctypes.c_int
    _lib = L
    return L


# exception text per status, as the reference throws them
MESSAGES = {
    MPDX_E_GRID: "libmpdata++: bogus grid size",
    MPDX_E_DIVERGENT: "libmpdata++: initial advector field is divergent",
    MPDX_E_PRS_STUCK: "libmpdata++: stuck in pressure solver",
}


class MpdxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code
