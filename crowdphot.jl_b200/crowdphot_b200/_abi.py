"""ctypes mirror of include/crowdphot_b200.h (structs, constants, prototypes).

The struct layouts here must match the C header field for field; the
`test_abi.py` suite checks every declared symbol and the struct sizes.
"""
from __future__ import annotations

import ctypes as C
import os

CPB_OK = 0
CPB_ERR_ARGUMENT = -1
CPB_ERR_CUDA = -2
CPB_ERR_OOM = -3
CPB_ERR_TIMEOUT = -4
CPB_FAULT_NONE = 0
CPB_FAULT_HOLD_READY_STAR = 1
CPB_ERR_INTERNAL = -5
CPB_ERR_NO_DEVICE = -6

CPB_F32 = 1
CPB_F64 = 2

CPB_PSF_GRIDDED_IMAGE = 1
CPB_PSF_IMAGE = 2
CPB_PSF_CIRCULAR_GAUSSIAN = 3

CPB_FREE_Y = 1
CPB_FREE_X = 2
CPB_FREE_FLUX = 4
CPB_FREE_BKG = 8
CPB_FREE_FWHM = 16

CPB_PREC_FP64 = 0
CPB_PREC_MIXED = 1

CPB_COV_AUTO = 0
CPB_COV_KNOWN_WEIGHTS = 1
CPB_COV_REWEIGHTED = 2

CPB_DAMP_MARQUARDT = 0
CPB_DAMP_LEVENBERG = 1
CPB_DAMP_NONE = 2

CPB_SOLVER_LSQR = 0
CPB_SOLVER_LSMR = 1

CPB_LOSS_NONE = 0
CPB_LOSS_L2DIST = 1
CPB_LOSS_HUBER = 2
CPB_LOSS_TUKEY = 3
CPB_LOSS_LOGITDIST = 4
CPB_SCALE_AUTO = 0
CPB_SCALE_MAD = 1
CPB_SCALE_FIXED = 2
CPB_SCALE_MSCALE = 3

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)


class PsfDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_nodes", C.c_int32),
        ("eltype", C.c_int32),
        ("reserved", C.c_int32),
        ("node_data", C.POINTER(C.c_void_p)),
        ("node_ny", _i64p),
        ("node_nx", _i64p),
        ("node_os", _i64p),
        ("node_origin", _dp),
        ("node_fill_value", _dp),
        ("grid_y", _dp),
        ("grid_x", _dp),
        ("fwhm", C.c_double),
    ]


class SimParams(C.Structure):
    _fields_ = [
        ("fit_rad", C.c_double),
        ("free_mask", C.c_int32),
        ("inner_iterations", C.c_int32),
        ("fixed_y", C.c_double),
        ("fixed_x", C.c_double),
        ("fixed_flux", C.c_double),
        ("fixed_bkg", C.c_double),
        ("fixed_fwhm", C.c_double),
        ("linear_tol", C.c_double),
        ("model_rad_auto", C.c_int32),
        ("max_trials", C.c_int32),
        ("model_rad", C.c_double),
        ("model_rad_max", C.c_double),
        ("model_rad_nsigma", C.c_double),
        ("max_step", C.c_double),
        ("max_iter", C.c_int32),
        ("covariance", C.c_int32),
        ("x_tol", C.c_double),
        ("f_tol", C.c_double),
        ("g_tol", C.c_double),
        ("lambda_init", C.c_double),
        ("lambda_up", C.c_double),
        ("lambda_down", C.c_double),
        ("lambda_min", C.c_double),
        ("lambda_max", C.c_double),
        ("precision", C.c_int32),
        ("solver", C.c_int32),
        ("damping", C.c_int32),
        ("refine_iters", C.c_int32),
        ("spread_model_fwhm", C.c_double),
    ]


class SimResult(C.Structure):
    _fields_ = [
        ("y", _dp), ("x", _dp), ("flux", _dp), ("bkg", _dp),
        ("y_err", _dp), ("x_err", _dp), ("flux_err", _dp), ("bkg_err", _dp),
        ("converged", _u8p), ("valid", _u8p),
        ("chisq", _dp),
        ("qfit", _dp), ("qfit_expected", _dp), ("qfit_z", _dp), ("crowding", _dp),
        ("n_iter", _i32p),
        ("residual", _dp),
        ("dbg_active", _i32p),
        ("dbg_pixels", _i32p),
        ("dbg_model_R", _i32p),
        ("n_passes", C.c_int32),
        ("n_failed", C.c_int32),
        ("n_active", C.c_int64),
        ("n_union", C.c_int64),
        ("n_trials", C.c_int64),
        ("n_lsqr_iters", C.c_int64),
        ("model_px_evals", C.c_double),
        ("lsqr_px_macs", C.c_double),
        ("device_seconds", C.c_double),
        ("spread_model", _dp), ("spread_model_err", _dp),
    ]


class MultipassResult(C.Structure):
    _fields_ = [
        ("params", _dp), ("errors", _dp),
        ("converged", _u8p), ("valid", _u8p),
        ("chisq", _dp),
        ("qfit", _dp), ("qfit_expected", _dp), ("qfit_z", _dp), ("crowding", _dp),
        ("n_iter", _i32p),
        ("residual", _dp),
        ("n_passes", C.c_int32), ("n_failed", C.c_int32),
        ("n_levels", C.c_int64), ("n_fits", C.c_int64),
        ("device_seconds", C.c_double),
        ("spread_model", _dp), ("spread_model_err", _dp),
    ]


class GroupResult(C.Structure):
    _fields_ = [
        ("y", _dp), ("x", _dp), ("flux", _dp),
        ("y_err", _dp), ("x_err", _dp), ("flux_err", _dp),
        ("converged", _u8p), ("valid", _u8p),
        ("n_iter", _i32p),
        ("chisq", _dp),
        ("qfit", _dp), ("qfit_expected", _dp), ("qfit_z", _dp), ("crowding", _dp),
        ("residual", _dp),
        ("n_passes", _i32p), ("n_failed", _i32p), ("status", _i32p),
        ("error_kind", _i32p),
        ("n_active", _i32p), ("n_union", _i32p),
        ("n_trials", _i32p), ("n_lsqr_iters", _i32p),
        ("n_kernel_groups", C.c_int64),
        ("n_routed_groups", C.c_int64),
        ("device_seconds", C.c_double),
        ("spread_model", _dp), ("spread_model_err", _dp),
    ]


class TuneInfo(C.Structure):
    _fields_ = [
        ("lm_blocks_per_sm", C.c_int32), ("lm_node_in_smem", C.c_int32),
        ("grp_threads", C.c_int32), ("grp_blocks_per_sm", C.c_int32),
        ("from_cache", C.c_int32), ("n_timed", C.c_int32),
        ("lm_ms", C.c_double), ("grp_ms", C.c_double),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight", C.c_int32), ("hbm_reserve_bytes", C.c_int64)]


class RequestInfo(C.Structure):
    _fields_ = [
        ("state", C.c_int32), ("status", C.c_int32), ("slot", C.c_int32), ("reserved", C.c_int32),
        ("est_bytes", C.c_int64),
        ("queued_seconds", C.c_double), ("run_seconds", C.c_double), ("latency_seconds", C.c_double),
        ("device_seconds", C.c_double),
        ("start_time", C.c_double), ("end_time", C.c_double),
        ("error", C.c_char * 256),
    ]


CPB_REQ_QUEUED, CPB_REQ_RUNNING, CPB_REQ_DONE, CPB_REQ_FAILED, CPB_REQ_CANCELLED = 0, 1, 2, 3, 4


class LMParams(C.Structure):
    _fields_ = [
        ("free_mask", C.c_int32),
        ("max_iter", C.c_int32),
        ("fixed_y", C.c_double),
        ("fixed_x", C.c_double),
        ("fixed_flux", C.c_double),
        ("fixed_bkg", C.c_double),
        ("fixed_fwhm", C.c_double),
        ("x_tol", C.c_double),
        ("f_tol", C.c_double),
        ("g_tol", C.c_double),
        ("lambda_init", C.c_double),
        ("lambda_up", C.c_double),
        ("lambda_down", C.c_double),
        ("lambda_min", C.c_double),
        ("lambda_max", C.c_double),
        ("min_diagonal", C.c_double),
        ("damping", C.c_int32),
        ("covariance", C.c_int32),
        ("precision", C.c_int32),
        ("reserved", C.c_int32),
        ("reweight", C.c_int32),
        ("scale_estimator", C.c_int32),
        ("loss_param", C.c_double),
        ("scale_value", C.c_double),
        ("mscale_delta", C.c_double),
        ("mscale_tol", C.c_double),
        ("mscale_max_iter", C.c_int32),
        ("reserved2", C.c_int32),
        ("weight_reset_tol", C.c_double),
    ]


class LMResultC(C.Structure):
    _fields_ = [
        ("params", _dp),
        ("cov", _dp),
        ("cost", _dp), ("cost_init", _dp), ("chisq", _dp), ("lambda_final", _dp),
        ("converged", _u8p), ("x_converged", _u8p), ("f_converged", _u8p), ("g_converged", _u8p),
        ("iterations", _i32p),
        ("status", _i32p),
        ("device_seconds", C.c_double),
        ("sigma_final", _dp),
    ]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("seconds", C.c_double), ("bytes", C.c_double)]


# Every entry point declared in include/crowdphot_b200.h: name -> (restype, argtypes)
PROTOTYPES = {
    "cpb_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "cpb_ctx_destroy": (C.c_int, [C.c_void_p]),
    "cpb_last_error": (C.c_char_p, [C.c_void_p]),
    "cpb_version": (C.c_char_p, []),
    "cpb_ctx_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "cpb_ctx_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int64]),
    "cpb_ctx_inject_fault": (C.c_int, [C.c_void_p, C.c_int32]),
    "cpb_ctx_kernel_stats": (C.c_int, [C.c_void_p, C.POINTER(KernelStat), C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int64), C.c_int]),
    "cpb_psf_upload": (C.c_int, [C.c_void_p, C.POINTER(PsfDesc), C.POINTER(C.c_void_p)]),
    "cpb_psf_free": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cpb_fit_simultaneous": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(SimParams), C.c_void_p, C.c_int32,
                                       C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, _dp, _dp, _dp,
                                       C.POINTER(SimResult)]),
    "cpb_fit_simultaneous_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(SimParams), C.c_void_p, C.c_int32,
                                              C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.POINTER(SimResult)]),
    "cpb_fit_simultaneous_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(SimParams), C.c_void_p,
                                                      C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                                      C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                      C.POINTER(SimResult)]),
    "cpb_fit_simultaneous_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(SimParams), C.c_int64, _i64p,
                                             _i32p, _i32p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, _i64p,
                                             _dp, _dp, _dp, C.POINTER(GroupResult)]),
    "cpb_fit_simultaneous_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(SimParams), C.c_int64,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_int64, C.POINTER(GroupResult)]),
    "cpb_batch_graph_create": (C.c_int, [C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                         C.c_void_p,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int64, C.c_void_p,
                                         C.c_int32, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(TuneInfo)]),
    "cpb_batch_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "cpb_batch_graph_destroy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cpb_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "cpb_server_add_psf": (C.c_int, [C.c_void_p, C.POINTER(PsfDesc), C.POINTER(C.c_int32)]),
    "cpb_server_submit": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(SimParams), C.c_void_p, C.c_int32, C.c_int64,
                                    C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, _dp, _dp, _dp,
                                    C.POINTER(SimResult), C.POINTER(C.c_int64)]),
    "cpb_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(RequestInfo)]),
    "cpb_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
    "cpb_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "cpb_server_destroy": (C.c_int, [C.c_void_p]),
    "cpb_server_last_error": (C.c_char_p, [C.c_void_p]),
    "cpb_fit_all_stars": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LMParams), C.c_double, C.c_int32,
                                    C.c_double, C.c_void_p,
                                    C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, _dp,
                                    C.POINTER(MultipassResult)]),
    "cpb_exp_disk_kernel": (C.c_int, [C.c_double, C.c_int32, _dp]),
    "cpb_fit_lm_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LMParams), C.c_int64, _i64p, _i32p, _i32p,
                                   _i32p, _i32p, C.c_void_p, C.c_int32, C.c_void_p, _dp, C.POINTER(LMResultC)]),
    "cpb_fit_lm_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LMParams), C.c_int64, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                          C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(LMResultC)]),
}

PACKAGE_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# CROWDPHOT_B200_LIB (as for the Julia binding) selects another build of the library
LIB_PATH = os.environ.get("CROWDPHOT_B200_LIB") or os.path.join(PACKAGE_DIR, "lib", "libcrowdphot_b200.so")
# the same library with every stamp and pixel index of the simultaneous fit
# tested against its buffer (a failed test skips the access and fails the call)
CHECKED_LIB_PATH = os.path.join(PACKAGE_DIR, "lib", "libcrowdphot_b200_checked.so")

_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Loads libcrowdphot_b200.so and binds every prototype.  Raises when absent:
    there is no CPU fallback for the product path."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libcrowdphot_b200.so not found at {p}; build it with __graft_entry__.build()")
    lib = C.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
