"""Host mirror of CrowdPhot's photometry entry points over the B200 C-ABI.

``fit_all_stars_simultaneous`` mirrors
src/photometry/psf_photometry_simultaneous.jl:953-981 (same positional
arguments, keyword names, defaults and ArgumentError texts) and returns a
``MultiPassPhotResult`` (psf_photometry_single.jl:99-122).  ``fit_star``
mirrors src/psf/psf_fitting.jl:229-250 and returns ``(best_model, LMResult)``
(levenberg_marquardt.jl:28-41).  ``fit_star_batch`` runs many independent
fit_star calls in one launch.

Differences from the Julia API, all deliberate:
  * the device computes in FP64 and results are returned as float64 arrays
    (Float32 cannot hold 1e-4 px at 2048 px);
  * ``background`` (image-shaped, optional) is subtracted on the device;
  * IRLS losses other than L2DistLoss / HuberLoss / TukeyLoss / LogitDistLoss and PSF types
    other than CircularGaussianPSF / ImagePSF / GriddedPSFModel{ImagePSF} raise
    ArgumentError -- there is no CPU fallback;
  * ``solver=:lsmr`` groups of the batched fitter run one by one through the
    full-field fit (the block-per-group kernel solves by LSQR);
  * a simultaneous fit whose first catalogue star has a non-finite position
    returns ``spread_model`` NaN where the reference's ``_spread_fwhm`` raises
    an InexactError.
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from dataclasses import dataclass

import numpy as np

from . import _abi
from .psf import (ArgumentError, CircularGaussianPSF, GriddedPSFModel, ImagePSF, replace_params)

_tls_lock = threading.Lock()


class CudaError(RuntimeError):
    pass


class Context:
    """A device context (cpb_ctx) with an upload cache for PSFs."""

    def __init__(self, device: int = 0, lib: str | None = None):
        """lib: path of another build of the library (for instance the checked
        build, lib/libcrowdphot_b200_checked.so); default the package's own."""
        self.lib = _abi.load_library(lib)
        h = C.c_void_p()
        rc = self.lib.cpb_ctx_create(int(device), C.byref(h))
        if rc != _abi.CPB_OK:
            raise CudaError(f"cpb_ctx_create(device={device}) failed with status {rc}")
        self.handle = h
        self.device = device
        self._psfs: dict[int, tuple] = {}

    def close(self):
        if self.handle:
            for _, (hp, _ref) in list(self._psfs.items()):
                self.lib.cpb_psf_free(self.handle, hp)
            self._psfs.clear()
            self.lib.cpb_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def error(self) -> str:
        return self.lib.cpb_last_error(self.handle).decode()

    def raise_for(self, rc: int, what: str):
        if rc == _abi.CPB_OK:
            return
        msg = self.error()
        if rc == _abi.CPB_ERR_ARGUMENT:
            raise ArgumentError(msg)
        if rc == _abi.CPB_ERR_OOM:
            raise MemoryError(f"{what}: {msg}")
        if rc == _abi.CPB_ERR_TIMEOUT:
            raise TimeoutError(f"{what}: {msg}")
        raise CudaError(f"{what} failed ({rc}): {msg}")

    def set_profiling(self, enable: bool):
        self.raise_for(self.lib.cpb_ctx_set_profiling(self.handle, int(bool(enable))), "cpb_ctx_set_profiling")

    def set_wait_limit(self, polls: int):
        """Polls (of >= 64 ns) a bounded device wait makes before the call gives up
        with CPB_ERR_TIMEOUT; <= 0 restores the default (2^26)."""
        self.raise_for(self.lib.cpb_ctx_set_wait_limit(self.handle, int(polls)), "cpb_ctx_set_wait_limit")

    def inject_fault(self, fault: int):
        """One-shot host-side fault injection for tests (CPB_FAULT_*)."""
        self.raise_for(self.lib.cpb_ctx_inject_fault(self.handle, int(fault)), "cpb_ctx_inject_fault")

    def kernel_stats(self, reset: bool = True):
        """Per-kernel launch counts, event-timed seconds and algorithmic bytes, plus
        the total launch count since the last reset."""
        buf = (_abi.KernelStat * 64)()
        n = C.c_int()
        launches = C.c_int64()
        rc = self.lib.cpb_ctx_kernel_stats(self.handle, buf, 64, C.byref(n), C.byref(launches), int(reset))
        self.raise_for(rc, "cpb_ctx_kernel_stats")
        stats = {buf[i].name.decode(): dict(launches=int(buf[i].launches), seconds=float(buf[i].seconds),
                                            bytes=float(buf[i].bytes)) for i in range(min(n.value, 64))}
        return stats, int(launches.value)

    def psf_handle(self, psf, fwhm_override=None):
        key = id(psf)
        hit = self._psfs.get(key)
        if hit is not None and hit[1]() is psf:
            return hit[0]
        desc, keep = psf_descriptor(psf)
        hp = C.c_void_p()
        rc = self.lib.cpb_psf_upload(self.handle, C.byref(desc), C.byref(hp))
        self.raise_for(rc, "cpb_psf_upload")
        del keep
        self._psfs[key] = (hp, weakref.ref(psf))
        return hp


_default_ctx: Context | None = None


def get_context(device: int = 0) -> Context:
    global _default_ctx
    with _tls_lock:
        if _default_ctx is None or _default_ctx.device != device:
            _default_ctx = Context(device)
        return _default_ctx


def psf_descriptor(psf):
    """Builds a cpb_psf_desc for a supported PSF; returns (desc, keepalive)."""
    d = _abi.PsfDesc()
    keep = []
    if isinstance(psf, CircularGaussianPSF):
        d.kind = _abi.CPB_PSF_CIRCULAR_GAUSSIAN
        d.n_nodes = 0
        d.eltype = _abi.CPB_F64
        d.fwhm = float(psf.fwhm)
        return d, keep
    if isinstance(psf, ImagePSF):
        nodes, gy, gx, kind = [psf], [0.0], [0.0], _abi.CPB_PSF_IMAGE
    elif isinstance(psf, GriddedPSFModel):
        nodes, gy, gx, kind = psf.psfs, list(psf.grid_y), list(psf.grid_x), _abi.CPB_PSF_GRIDDED_IMAGE
    else:
        raise ArgumentError(f"unsupported PSF type {type(psf).__name__} for the B200 path")
    n = len(nodes)
    datas = [np.asfortranarray(nd.data, dtype=np.float64) for nd in nodes]
    keep += datas
    ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in datas])
    ny = np.array([a.shape[0] for a in datas], dtype=np.int64)
    nx = np.array([a.shape[1] for a in datas], dtype=np.int64)
    os_ = np.array([v for nd in nodes for v in nd.oversampling], dtype=np.int64)
    org = np.array([v for nd in nodes for v in (nd.origin["y"], nd.origin["x"])], dtype=np.float64)
    fill = np.array([nd.fill_value for nd in nodes], dtype=np.float64)
    gya = np.asarray(gy, dtype=np.float64)
    gxa = np.asarray(gx, dtype=np.float64)
    keep += [ptrs, ny, nx, os_, org, fill, gya, gxa]
    d.kind = kind
    d.n_nodes = n
    d.eltype = _abi.CPB_F64
    d.node_data = C.cast(ptrs, C.POINTER(C.c_void_p))
    d.node_ny = ny.ctypes.data_as(_abi._i64p)
    d.node_nx = nx.ctypes.data_as(_abi._i64p)
    d.node_os = os_.ctypes.data_as(_abi._i64p)
    d.node_origin = org.ctypes.data_as(_abi._dp)
    d.node_fill_value = fill.ctypes.data_as(_abi._dp)
    d.grid_y = gya.ctypes.data_as(_abi._dp)
    d.grid_x = gxa.ctypes.data_as(_abi._dp)
    return d, keep


@dataclass
class MultiPassPhotResult:
    """MultiPassPhotResult (psf_photometry_single.jl:99-122)."""
    y: np.ndarray
    x: np.ndarray
    y_err: np.ndarray
    x_err: np.ndarray
    flux: np.ndarray
    flux_err: np.ndarray
    bkg: np.ndarray
    bkg_err: np.ndarray
    converged: np.ndarray
    valid: np.ndarray
    chisq: np.ndarray
    qfit: np.ndarray
    qfit_expected: np.ndarray
    qfit_z: np.ndarray
    crowding: np.ndarray
    spread_model: np.ndarray
    spread_model_err: np.ndarray
    n_iter: np.ndarray
    n_passes: int
    n_failed: int
    failure_msgs: list
    residual: np.ndarray
    stats: dict | None = None
    debug: dict | None = None


@dataclass
class LMResult:
    """LMResult (levenberg_marquardt.jl:28-41)."""
    minimizer: np.ndarray
    minimum: float
    cost_init: float
    converged: bool
    x_converged: bool
    f_converged: bool
    g_converged: bool
    iterations: int
    lambda_final: float
    sigma_final: float
    cov: np.ndarray
    chisq: float


_DAMPING = {"marquardt": _abi.CPB_DAMP_MARQUARDT, "levenberg": _abi.CPB_DAMP_LEVENBERG,
            "none": _abi.CPB_DAMP_NONE}
_COV = {None: _abi.CPB_COV_AUTO, "known_weights": _abi.CPB_COV_KNOWN_WEIGHTS,
        "reweighted": _abi.CPB_COV_REWEIGHTED}
_PREC = {"fp64": _abi.CPB_PREC_FP64, "mixed": _abi.CPB_PREC_MIXED}


def _props(psf):
    if isinstance(psf, CircularGaussianPSF):
        return ("y", "x", "fwhm", "flux", "bkg")
    if isinstance(psf, (ImagePSF, GriddedPSFModel)):
        return ("y", "x", "flux", "bkg")
    raise ArgumentError(f"unsupported PSF type {type(psf).__name__} for the B200 path")


_BITS = {"y": _abi.CPB_FREE_Y, "x": _abi.CPB_FREE_X, "flux": _abi.CPB_FREE_FLUX, "bkg": _abi.CPB_FREE_BKG,
         "fwhm": _abi.CPB_FREE_FWHM}


def _free_mask(psf, fixed):
    mask = 0
    for k in _props(psf):
        if k not in fixed:
            mask |= _BITS[k]
    return mask


def _image_arrays(image, inv_var, background):
    img = np.asarray(image)
    if img.ndim != 2:
        raise ArgumentError("`image` must be a matrix")
    dt = np.float32 if img.dtype == np.float32 else np.float64
    imgf = np.asfortranarray(img, dtype=dt)
    ivf = None
    if inv_var is not None:
        iv = np.asarray(inv_var)
        if iv.shape != img.shape:
            raise ArgumentError("`inv_var` must be the same size as `image`")
        ivf = np.asfortranarray(iv, dtype=dt)
    bkf = None
    if background is not None:
        bk = np.asarray(background)
        if bk.ndim == 0:
            bk = np.full(img.shape, float(bk))
        if bk.shape != img.shape:
            raise ArgumentError("`background` must be the same size as `image`")
        bkf = np.asfortranarray(bk, dtype=dt)
    et = _abi.CPB_F32 if dt == np.float32 else _abi.CPB_F64
    return imgf, ivf, bkf, et


def _catalog(sources):
    """_extract_source_catalog for NamedTuple-like catalogues (psf_photometry_single.jl:167-181)."""
    get = (lambda k: sources[k]) if isinstance(sources, dict) else (lambda k: getattr(sources, k))
    has = (lambda k: k in sources) if isinstance(sources, dict) else (lambda k: hasattr(sources, k))
    y = np.ascontiguousarray(np.asarray(get("y"), dtype=np.float64).ravel())
    x = np.ascontiguousarray(np.asarray(get("x"), dtype=np.float64).ravel())
    n = y.size
    f = np.ascontiguousarray(np.asarray(get("flux"), dtype=np.float64).ravel()) if has("flux") else np.ones(n)
    if x.size != n or f.size != n:
        raise ArgumentError("source y/x/flux lengths must match")
    return y, x, f


def sim_params(psf, fit_rad, fixed, *, inv_var_given, solver="lsqr", inner_iterations=10, linear_tol=1.0e-6,
               model_rad="auto", model_rad_max=None, model_rad_nsigma=1.0, max_step=0.25, max_trials=8, max_iter=40,
               x_tol=1.0e-5, f_tol=1.0e-4, g_tol=1.0e-4, lambda_init=1.0e-4, lambda_up=10.0, lambda_down=10.0,
               lambda_min=1.0e-12, lambda_max=1.0e12, damping="marquardt", covariance_estimator=None,
               precision="fp64", spread_model_fwhm=None, refine_iters=0):
    """Keyword arguments -> cpb_sim_params (shared by the device path and the oracle).

    refine_iters (precision="mixed" only): FP64 Gauss-Newton iterations after the
    FP32-stamp loop, every active star live again from the mixed-precision
    parameters and the damping restarted at lambda_init; 0 keeps the
    mixed-precision parameters and re-evaluates only the errors, residual and
    diagnostics in FP64."""
    P = _abi.SimParams()
    P.spread_model_fwhm = spread_fwhm_arg(spread_model_fwhm)
    P.fit_rad = float(fit_rad)
    P.free_mask = _free_mask(psf, fixed)
    P.inner_iterations = int(inner_iterations)
    P.fixed_y = float(fixed.get("y", 0.0))
    P.fixed_x = float(fixed.get("x", 0.0))
    P.fixed_flux = float(fixed.get("flux", 1.0))
    P.fixed_bkg = float(fixed.get("bkg", 0.0))
    P.fixed_fwhm = float(fixed.get("fwhm", getattr(psf, "fwhm", 0.0)))
    P.linear_tol = float(linear_tol)
    if isinstance(model_rad, str):
        if model_rad != "auto":
            raise ArgumentError(f"model_rad must be :auto or a positive real, got :{model_rad}")
        P.model_rad_auto = 1
        P.model_rad = 0.0
    else:
        P.model_rad_auto = 0
        P.model_rad = float(model_rad)
    P.max_trials = int(max_trials)
    P.model_rad_max = float(10 * fit_rad if model_rad_max is None else model_rad_max)
    P.model_rad_nsigma = float(model_rad_nsigma)
    P.max_step = float(max_step)
    P.max_iter = int(max_iter)
    P.covariance = _COV[covariance_estimator]
    P.x_tol, P.f_tol, P.g_tol = float(x_tol), float(f_tol), float(g_tol)
    P.lambda_init, P.lambda_up, P.lambda_down = float(lambda_init), float(lambda_up), float(lambda_down)
    P.lambda_min, P.lambda_max = float(lambda_min), float(lambda_max)
    P.precision = _PREC[precision]
    if int(refine_iters) < 0:
        raise ArgumentError("refine_iters must be >= 0")
    P.refine_iters = int(refine_iters)
    if solver not in ("lsqr", "lsmr"):
        raise ArgumentError(f"solver must be :lsqr or :lsmr, got :{solver}")
    P.solver = _abi.CPB_SOLVER_LSQR if solver == "lsqr" else _abi.CPB_SOLVER_LSMR
    P.damping = _DAMPING[damping]
    return P


def spread_fwhm_arg(v):
    """spread_model_fwhm keyword -> the C-ABI double: nothing (None) -> NaN, the
    PSF-derived width; a non-finite or non-positive value -> 0, no spread_model
    (the reference skips the reference disk when the width is not finite and > 0)."""
    if v is None:
        return float("nan")
    v = float(v)
    return v if np.isfinite(v) and v > 0 else 0.0


class SimOutputs:
    """Caller-owned output arrays for one cpb_sim_result."""

    def __init__(self, n, ny, nx, S2, residual=True, debug=False):
        self.n = n
        z = lambda: np.zeros(max(n, 1), dtype=np.float64)
        self.y, self.x, self.flux, self.bkg = z(), z(), z(), z()
        self.y_err, self.x_err, self.flux_err, self.bkg_err = z(), z(), z(), z()
        self.chisq, self.qfit, self.qfit_expected, self.qfit_z, self.crowding = z(), z(), z(), z(), z()
        self.spread_model, self.spread_model_err = z(), z()
        self.converged = np.zeros(max(n, 1), dtype=np.uint8)
        self.valid = np.zeros(max(n, 1), dtype=np.uint8)
        self.n_iter = np.zeros(max(n, 1), dtype=np.int32)
        self.residual = np.zeros((ny, nx), dtype=np.float64, order="F") if residual else None
        self.debug = debug
        if debug:
            self.dbg_active = np.full(max(n, 1), -1, dtype=np.int32)
            self.dbg_pixels = np.zeros(max(S2 * n, 1), dtype=np.int32)
            self.dbg_model_R = np.zeros(max(n, 1), dtype=np.int32)
        r = _abi.SimResult()
        dp = lambda a: a.ctypes.data_as(_abi._dp)
        r.y, r.x, r.flux, r.bkg = dp(self.y), dp(self.x), dp(self.flux), dp(self.bkg)
        r.y_err, r.x_err, r.flux_err, r.bkg_err = dp(self.y_err), dp(self.x_err), dp(self.flux_err), dp(self.bkg_err)
        r.converged = self.converged.ctypes.data_as(_abi._u8p)
        r.valid = self.valid.ctypes.data_as(_abi._u8p)
        r.chisq, r.qfit, r.qfit_expected = dp(self.chisq), dp(self.qfit), dp(self.qfit_expected)
        r.qfit_z, r.crowding = dp(self.qfit_z), dp(self.crowding)
        r.spread_model, r.spread_model_err = dp(self.spread_model), dp(self.spread_model_err)
        r.n_iter = self.n_iter.ctypes.data_as(_abi._i32p)
        if residual:
            r.residual = dp(self.residual)
        if debug:
            r.dbg_active = self.dbg_active.ctypes.data_as(_abi._i32p)
            r.dbg_pixels = self.dbg_pixels.ctypes.data_as(_abi._i32p)
            r.dbg_model_R = self.dbg_model_R.ctypes.data_as(_abi._i32p)
        self.c = r

    def result(self, ny, nx, S2) -> MultiPassPhotResult:
        n = self.n
        r = self.c
        valid = self.valid[:n].astype(bool)
        msgs = []
        if r.n_active < n:
            msgs = [f"star {i + 1}: excluded before the solve (no usable pixels or non-finite initial parameters)"
                    for i in np.flatnonzero(~valid).tolist()]
        res = MultiPassPhotResult(
            y=self.y[:n].copy(), x=self.x[:n].copy(), y_err=self.y_err[:n].copy(), x_err=self.x_err[:n].copy(),
            flux=self.flux[:n].copy(), flux_err=self.flux_err[:n].copy(), bkg=self.bkg[:n].copy(),
            bkg_err=self.bkg_err[:n].copy(), converged=self.converged[:n].astype(bool), valid=valid,
            chisq=self.chisq[:n].copy(), qfit=self.qfit[:n].copy(), qfit_expected=self.qfit_expected[:n].copy(),
            qfit_z=self.qfit_z[:n].copy(), crowding=self.crowding[:n].copy(),
            spread_model=self.spread_model[:n].copy(), spread_model_err=self.spread_model_err[:n].copy(),
            n_iter=self.n_iter[:n].astype(np.int64), n_passes=int(r.n_passes),
            n_failed=int(r.n_failed), failure_msgs=msgs,
            residual=self.residual if self.residual is not None else np.zeros((ny, nx)),
            stats=dict(n_active=int(r.n_active), n_union=int(r.n_union), n_trials=int(r.n_trials),
                       n_lsqr_iters=int(r.n_lsqr_iters), model_px_evals=float(r.model_px_evals),
                       lsqr_px_macs=float(r.lsqr_px_macs), device_seconds=float(r.device_seconds)))
        if self.debug:
            na = int(r.n_active)
            res.debug = dict(active=self.dbg_active[:na].copy(),
                             pixels=self.dbg_pixels[:S2 * na].reshape(na, S2).copy(),
                             model_R=self.dbg_model_R[:na].copy())
        return res


def fit_all_stars_simultaneous(image, psf, sources, fit_rad, *, fixed=None, inv_var=None, background=None,
                               spread_model_fwhm=None, solver="lsqr", inner_iterations=10, linear_tol=1.0e-6,
                               model_rad="auto", model_rad_max=None, model_rad_nsigma=1.0, max_step=0.25,
                               max_trials=8, max_iter=40, x_tol=1.0e-5, f_tol=1.0e-4, g_tol=1.0e-4,
                               lambda_init=1.0e-4, lambda_up=10.0, lambda_down=10.0, lambda_min=1.0e-12,
                               lambda_max=1.0e12, damping="marquardt", show_trace=False, covariance_estimator=None,
                               precision="fp64", refine_iters=0, ctx: Context | None = None, debug=False,
                               residual=True) -> MultiPassPhotResult:
    """CrowdPhot.fit_all_stars_simultaneous on the B200 (psf_photometry_simultaneous.jl:953-1431)."""
    fixed = dict(fixed or {})
    ctx = ctx or get_context()
    imgf, ivf, bkf, et = _image_arrays(image, inv_var, background)
    y0, x0, f0 = _catalog(sources)
    P = sim_params(psf, fit_rad, fixed, inv_var_given=ivf is not None, solver=solver,
                   inner_iterations=inner_iterations, linear_tol=linear_tol, model_rad=model_rad,
                   model_rad_max=model_rad_max, model_rad_nsigma=model_rad_nsigma, max_step=max_step,
                   max_trials=max_trials, max_iter=max_iter, x_tol=x_tol, f_tol=f_tol, g_tol=g_tol,
                   lambda_init=lambda_init, lambda_up=lambda_up, lambda_down=lambda_down, lambda_min=lambda_min,
                   lambda_max=lambda_max, damping=damping, covariance_estimator=covariance_estimator,
                   precision=precision, spread_model_fwhm=spread_model_fwhm, refine_iters=refine_iters)
    ny, nx = imgf.shape
    R = int(np.ceil(fit_rad)) if fit_rad > 0 else 0
    S2 = (2 * R + 1) ** 2
    outs = SimOutputs(y0.size, ny, nx, S2, residual=residual, debug=debug)
    hp = ctx.psf_handle(psf)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.cpb_fit_simultaneous(ctx.handle, hp, C.byref(P), vp(imgf), et, ny, nx, vp(ivf), vp(bkf),
                                      y0.size, y0.ctypes.data_as(_abi._dp), x0.ctypes.data_as(_abi._dp),
                                      f0.ctypes.data_as(_abi._dp), C.byref(outs.c))
    ctx.raise_for(rc, "cpb_fit_simultaneous")
    return outs.result(ny, nx, S2)


_GROUP_ERRORS = {
    1: "the image contains non-finite values but `inv_var` was not provided; pass `inv_var` to mask them or clean "
       "the image first",
    2: "InexactError: a star's integer anchor is negative (Morton key of a negative coordinate)",
}


def group_outputs(n_stars, n_groups, total_pixels=0, residual=False):
    """Caller-owned output arrays of one cpb_group_result (numpy, host)."""
    ns, G = max(n_stars, 1), max(n_groups, 1)
    o = {k: np.zeros(ns) for k in ("y", "x", "flux", "y_err", "x_err", "flux_err", "chisq", "qfit",
                                   "qfit_expected", "qfit_z", "crowding", "spread_model", "spread_model_err")}
    o.update(converged=np.zeros(ns, np.uint8), valid=np.zeros(ns, np.uint8), n_iter=np.zeros(ns, np.int32))
    o.update({k: np.zeros(G, np.int32) for k in ("n_passes", "n_failed", "status", "error_kind", "n_active",
                                                 "n_union", "n_trials", "n_lsqr_iters")})
    if residual:
        o["residual"] = np.zeros(max(total_pixels, 1))
    return o


def group_result_struct(o, ptr):
    """cpb_group_result over the arrays of `o`; ptr(array) gives its address (host or device)."""
    r = _abi.GroupResult()
    for name, _ in _abi.GroupResult._fields_:
        if name in o:
            setattr(r, name, C.cast(C.c_void_p(ptr(o[name])), dict(_abi.GroupResult._fields_)[name]))
    return r


def fit_groups_packed(psf, pixels, offsets, ny, nx, star_offsets, y0, x0, flux0, fit_rad, *, inv_var=None,
                      background=None, fixed=None, ctx: Context | None = None, residual=False, **kw):
    """Many independent fit_all_stars_simultaneous calls in one batch, packed form.

    Group g's image is the column-major block pixels[offsets[g] : offsets[g] + ny[g]*nx[g]] (inv_var and
    background share the layout); its catalogue is y0/x0/flux0[star_offsets[g] : star_offsets[g+1]] in the
    group's own 1-based coordinates.  Returns the per-star and per-group output arrays of cpb_group_result
    plus the batch counters.  Keyword arguments are those of fit_all_stars_simultaneous."""
    fixed = dict(fixed or {})
    ctx = ctx or get_context()
    pix = np.ascontiguousarray(pixels)
    dt = np.float32 if pix.dtype == np.float32 else np.float64
    pix = np.ascontiguousarray(pix, dtype=dt)
    iv = None if inv_var is None else np.ascontiguousarray(inv_var, dtype=dt)
    bk = None if background is None else np.ascontiguousarray(background, dtype=dt)
    et = _abi.CPB_F32 if dt == np.float32 else _abi.CPB_F64
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    nyv = np.ascontiguousarray(ny, dtype=np.int32)
    nxv = np.ascontiguousarray(nx, dtype=np.int32)
    so = np.ascontiguousarray(star_offsets, dtype=np.int64)
    G = off.size
    if nyv.size != G or nxv.size != G or so.size != G + 1:
        raise ArgumentError("offsets, ny, nx must have one entry per group and star_offsets one more")
    ys, xs, fs = (np.ascontiguousarray(a, dtype=np.float64) for a in (y0, x0, flux0))
    if not (ys.size == xs.size == fs.size == (so[-1] if G else 0)):
        raise ArgumentError("catalogue lengths must equal star_offsets[end]")
    P = sim_params(psf, fit_rad, fixed, inv_var_given=iv is not None, **kw)
    o = group_outputs(int(ys.size), G, int(pix.size), residual=residual)
    r = group_result_struct(o, lambda a: a.ctypes.data)
    hp = ctx.psf_handle(psf)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.cpb_fit_simultaneous_batch(ctx.handle, hp, C.byref(P), G, off.ctypes.data_as(_abi._i64p),
                                            nyv.ctypes.data_as(_abi._i32p), nxv.ctypes.data_as(_abi._i32p), vp(pix),
                                            et, vp(iv), vp(bk), so.ctypes.data_as(_abi._i64p),
                                            ys.ctypes.data_as(_abi._dp), xs.ctypes.data_as(_abi._dp),
                                            fs.ctypes.data_as(_abi._dp), C.byref(r))
    ctx.raise_for(rc, "cpb_fit_simultaneous_batch")
    ns = int(ys.size)
    res = {k: (v[:ns] if v.size >= ns and k not in ("n_passes", "n_failed", "status", "error_kind", "n_active",
                                                     "n_union", "n_trials", "n_lsqr_iters", "residual") else v)
           for k, v in o.items()}
    for k in ("n_passes", "n_failed", "status", "error_kind", "n_active", "n_union", "n_trials", "n_lsqr_iters"):
        res[k] = o[k][:G]
    res.update(n_kernel_groups=int(r.n_kernel_groups), n_routed_groups=int(r.n_routed_groups),
               device_seconds=float(r.device_seconds))
    return res


def fit_all_stars_simultaneous_batch(images, psf, sources_list, fit_rad, *, inv_vars=None, backgrounds=None,
                                     fixed=None, ctx: Context | None = None, residual=True,
                                     **kw) -> list[MultiPassPhotResult]:
    """fit_all_stars_simultaneous on each (image, sources) pair, all in one batch
    (psf_photometry_simultaneous.jl:953-1431 per group).  A group that fails the
    reference's data checks raises its ArgumentError, as the single call would."""
    G = len(images)
    if len(sources_list) != G:
        raise ArgumentError("one catalogue per image is required")
    arrs = [_image_arrays(im, None if inv_vars is None else inv_vars[g],
                          None if backgrounds is None else backgrounds[g]) for g, im in enumerate(images)]
    ets = {a[3] for a in arrs}
    if len(ets) > 1:
        raise ArgumentError("all images of a batch must share one element type")
    if inv_vars is not None and any(a[1] is None for a in arrs):
        raise ArgumentError("inv_vars must give one array per image")
    cats = [_catalog(s) for s in sources_list]
    sizes = np.array([a[0].size for a in arrs], np.int64)
    offs = np.zeros(G, np.int64)
    offs[1:] = np.cumsum(sizes)[:-1]
    flat = lambda k: np.concatenate([a[k].ravel(order="F") for a in arrs]) if G else np.zeros(0)
    pix = flat(0)
    iv = flat(1) if inv_vars is not None else None
    bk = flat(2) if backgrounds is not None else None
    so = np.zeros(G + 1, np.int64)
    so[1:] = np.cumsum([c[0].size for c in cats])
    cat = lambda k: np.concatenate([c[k] for c in cats]) if G else np.zeros(0)
    out = fit_groups_packed(psf, pix, offs, [a[0].shape[0] for a in arrs], [a[0].shape[1] for a in arrs], so,
                            cat(0), cat(1), cat(2), fit_rad, inv_var=iv, background=bk, fixed=fixed, ctx=ctx,
                            residual=residual, **kw)
    fixed = dict(fixed or {})
    results = []
    for g in range(G):
        if out["status"][g] != 0:
            raise ArgumentError(_GROUP_ERRORS.get(int(out["error_kind"][g]), "invalid group input"))
        s0, s1 = so[g], so[g + 1]
        n = int(s1 - s0)
        sl = slice(s0, s1)
        ny_, nx_ = arrs[g][0].shape
        valid = out["valid"][sl].astype(bool)
        msgs = [] if out["n_active"][g] == n else [
            f"star {i + 1}: excluded before the solve (no usable pixels or non-finite initial parameters)"
            for i in range(n) if not valid[i]]
        resid = (out["residual"][offs[g]:offs[g] + sizes[g]].reshape((ny_, nx_), order="F").copy()
                 if residual else np.zeros((ny_, nx_)))
        results.append(MultiPassPhotResult(
            y=out["y"][sl].copy(), x=out["x"][sl].copy(), y_err=out["y_err"][sl].copy(),
            x_err=out["x_err"][sl].copy(), flux=out["flux"][sl].copy(), flux_err=out["flux_err"][sl].copy(),
            bkg=np.full(n, float(fixed.get("bkg", 0.0))), bkg_err=np.zeros(n),
            converged=out["converged"][sl].astype(bool), valid=valid, chisq=out["chisq"][sl].copy(),
            qfit=out["qfit"][sl].copy(), qfit_expected=out["qfit_expected"][sl].copy(),
            qfit_z=out["qfit_z"][sl].copy(), crowding=out["crowding"][sl].copy(),
            spread_model=out["spread_model"][sl].copy(), spread_model_err=out["spread_model_err"][sl].copy(),
            n_iter=out["n_iter"][sl].astype(np.int64),
            n_passes=int(out["n_passes"][g]), n_failed=int(out["n_failed"][g]), failure_msgs=msgs, residual=resid,
            stats=dict(n_active=int(out["n_active"][g]), n_union=int(out["n_union"][g]),
                       n_trials=int(out["n_trials"][g]), n_lsqr_iters=int(out["n_lsqr_iters"][g]),
                       batch_device_seconds=out["device_seconds"])))
    return results


class BatchGraph:
    """One captured CUDA graph that fits a batch of fit_star cutouts and a batch of
    star groups concurrently (cpb_batch_graph_*).  Inputs and outputs are torch
    tensors on the context's device, bound at construction: refill the inputs in
    place and call launch() again.  `lm` holds the fit_star half
    (offsets, ny, nx, y1, x1, pix, inv_var, init and the _lm_outputs tensors under
    `out`), `groups` the group half (offsets, ny, nx, pix, inv_var, background,
    star_offsets, y, x, flux and the group_outputs tensors under `out`); either
    may be None.  autotune: 0 defaults, 1 tuned shapes (cached in cache_path),
    2 re-tune."""

    def __init__(self, psf, *, lm=None, lm_fixed=None, groups=None, fit_rad=None, group_kw=None,
                 autotune=1, cache_path=None, ctx: Context | None = None):
        self.ctx = ctx or get_context()
        self._keep = []
        hp = self.ctx.psf_handle(psf)
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        lm_args = [None, 0] + [None] * 6 + [0, None, None, 0, None]
        if lm is not None:
            P = lm_params(psf, dict(lm_fixed or {}))
            r = _lm_result_struct(lm["out"], lambda a: a.data_ptr())
            self._keep += [P, r]
            et = _abi.CPB_F32 if str(lm["pix"].dtype) == "torch.float32" else _abi.CPB_F64
            lm_args = [C.byref(P), int(lm["ny"].numel()), ptr(lm["offsets"]), ptr(lm["ny"]), ptr(lm["nx"]),
                       ptr(lm["y1"]), ptr(lm["x1"]), ptr(lm["pix"]), et, ptr(lm.get("inv_var")), ptr(lm["init"]),
                       int(lm["pix"].numel()), C.byref(r)]
        g_args = [None, 0] + [None] * 4 + [0] + [None] * 6 + [0, None]
        if groups is not None:
            kw = dict(group_kw or {})
            fixed = dict(kw.pop("fixed", {}) or {})
            SP = sim_params(psf, fit_rad, fixed, inv_var_given=groups.get("inv_var") is not None, **kw)
            gr = group_result_struct(groups["out"], lambda a: a.data_ptr())
            self._keep += [SP, gr]
            et = _abi.CPB_F32 if str(groups["pix"].dtype) == "torch.float32" else _abi.CPB_F64
            g_args = [C.byref(SP), int(groups["ny"].numel()), ptr(groups["offsets"]), ptr(groups["ny"]),
                      ptr(groups["nx"]), ptr(groups["pix"]), et, ptr(groups.get("inv_var")),
                      ptr(groups.get("background")), ptr(groups["star_offsets"]), ptr(groups["y"]), ptr(groups["x"]),
                      ptr(groups["flux"]), int(groups["pix"].numel()), C.byref(gr)]
        self.handle = C.c_void_p()
        self.info = _abi.TuneInfo()
        rc = self.ctx.lib.cpb_batch_graph_create(self.ctx.handle, hp, *lm_args, *g_args, int(autotune),
                                                 None if cache_path is None else str(cache_path).encode(),
                                                 C.byref(self.handle), C.byref(self.info))
        self.ctx.raise_for(rc, "cpb_batch_graph_create")
        self.lm, self.groups = lm, groups

    def launch(self) -> float:
        """Replays the graph; returns its device time in seconds."""
        t = C.c_double()
        rc = self.ctx.lib.cpb_batch_graph_launch(self.ctx.handle, self.handle, C.byref(t))
        self.ctx.raise_for(rc, "cpb_batch_graph_launch")
        return float(t.value)

    def tune_info(self) -> dict:
        return {k: getattr(self.info, k) for k, _ in _abi.TuneInfo._fields_}

    def close(self):
        if self.handle:
            self.ctx.lib.cpb_batch_graph_destroy(self.ctx.handle, self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Request:
    """A submitted fit (Server.submit): poll() / wait() / result() / cancel()."""

    _STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}

    def __init__(self, server, rid, keep, outs, shape):
        self.server, self.id, self._keep, self._outs, self._shape = server, rid, keep, outs, shape

    def _info(self, info):
        d = {k: getattr(info, k) for k, _ in _abi.RequestInfo._fields_ if k not in ("error", "reserved")}
        d["state"] = self._STATES.get(info.state, str(info.state))
        d["error"] = info.error.decode(errors="replace")
        return d

    def poll(self) -> dict:
        info = _abi.RequestInfo()
        self.server._check(self.server.lib.cpb_server_poll(self.server.handle, self.id, C.byref(info)), "poll")
        return self._info(info)

    def wait(self, timeout=None) -> dict:
        info = _abi.RequestInfo()
        rc = self.server.lib.cpb_server_wait(self.server.handle, self.id, -1.0 if timeout is None else float(timeout),
                                             C.byref(info))
        if rc == _abi.CPB_ERR_TIMEOUT:
            raise TimeoutError(f"request {self.id} still {self._STATES.get(info.state)} after {timeout} s")
        self.server._check(rc, "wait")
        return self._info(info)

    def result(self, timeout=None) -> MultiPassPhotResult:
        info = self.wait(timeout)
        if info["state"] == "cancelled":
            raise RuntimeError(f"request {self.id} was cancelled")
        if info["status"] != 0:
            if info["status"] == _abi.CPB_ERR_ARGUMENT:
                raise ArgumentError(info["error"])
            raise CudaError(f"request {self.id} failed ({info['status']}): {info['error']}")
        ny, nx, S2 = self._shape
        res = self._outs.result(ny, nx, S2)
        res.stats = dict(res.stats or {}, serving=info)
        return res

    def cancel(self) -> bool:
        return self.server.lib.cpb_server_cancel(self.server.handle, self.id) == 0


class Server:
    """Continuous batching of fit_all_stars_simultaneous requests on one GPU
    (cpb_server_*): up to `max_inflight` fits run at once on their own streams,
    admitted as slots and device memory free up; PSFs stay resident."""

    def __init__(self, device: int = 0, max_inflight: int = 4, hbm_reserve_bytes: int = -1):
        self.lib = _abi.load_library()
        cfg = _abi.ServerConfig(device, max_inflight, hbm_reserve_bytes)
        self.handle = C.c_void_p()
        rc = self.lib.cpb_server_create(C.byref(cfg), C.byref(self.handle))
        if rc != 0:
            raise CudaError(f"cpb_server_create failed ({rc})")
        self._psfs = {}

    def _check(self, rc, what):
        if rc == 0:
            return
        msg = (self.lib.cpb_server_last_error(self.handle) or b"").decode()
        if rc == _abi.CPB_ERR_ARGUMENT:
            raise ArgumentError(msg or what)
        raise CudaError(f"cpb_server_{what} failed ({rc}): {msg}")

    def psf_id(self, psf) -> int:
        key = id(psf)
        if key not in self._psfs:
            desc, keep = psf_descriptor(psf)
            pid = C.c_int32()
            self._check(self.lib.cpb_server_add_psf(self.handle, C.byref(desc), C.byref(pid)), "add_psf")
            del keep
            self._psfs[key] = (int(pid.value), psf)
        return self._psfs[key][0]

    def submit(self, image, psf, sources, fit_rad, *, fixed=None, inv_var=None, background=None, residual=False,
               **kw) -> Request:
        """Queues fit_all_stars_simultaneous(image, psf, sources, fit_rad; kw...) and returns at once."""
        fixed = dict(fixed or {})
        imgf, ivf, bkf, et = _image_arrays(image, inv_var, background)
        y0, x0, f0 = _catalog(sources)
        P = sim_params(psf, fit_rad, fixed, inv_var_given=ivf is not None, **kw)
        ny, nx = imgf.shape
        R = int(np.ceil(fit_rad)) if fit_rad > 0 else 0
        S2 = (2 * R + 1) ** 2
        outs = SimOutputs(y0.size, ny, nx, S2, residual=residual)
        pid = self.psf_id(psf)
        rid = C.c_int64()
        vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        self._check(self.lib.cpb_server_submit(self.handle, pid, C.byref(P), vp(imgf), et, ny, nx, vp(ivf), vp(bkf),
                                               y0.size, y0.ctypes.data_as(_abi._dp), x0.ctypes.data_as(_abi._dp),
                                               f0.ctypes.data_as(_abi._dp), C.byref(outs.c), C.byref(rid)), "submit")
        return Request(self, int(rid.value), (imgf, ivf, bkf, y0, x0, f0, P), outs, (ny, nx, S2))

    def close(self):
        if self.handle:
            self.lib.cpb_server_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lm_params(model, fixed, *, lambda_init=1.0e-4, lambda_up=10.0, lambda_down=10.0, lambda_min=1.0e-12,
              lambda_max=1.0e12, damping="marquardt", max_iter=200, x_tol=1.0e-8, f_tol=1.0e-4, g_tol=1.0e-4,
              covariance_estimator=None, min_diagonal=1.0e-6, precision="fp64", reweight=None, scale_estimator=None,
              weight_reset_tol=0.1, show_trace=False):
    """fit_star / lm_irls keyword arguments -> cpb_lm_params (psf_fitting.jl:229-250,
    levenberg_marquardt.jl:431-449); show_trace is accepted and ignored."""
    from .robust import set_irls
    P = _abi.LMParams()
    set_irls(P, reweight, scale_estimator, weight_reset_tol)
    P.free_mask = _free_mask(model, fixed)
    P.max_iter = int(max_iter)
    P.fixed_y = float(fixed.get("y", model.y))
    P.fixed_x = float(fixed.get("x", model.x))
    P.fixed_flux = float(fixed.get("flux", model.flux))
    P.fixed_bkg = float(fixed.get("bkg", model.bkg))
    P.fixed_fwhm = float(fixed.get("fwhm", getattr(model, "fwhm", 0.0)))
    P.x_tol, P.f_tol, P.g_tol = float(x_tol), float(f_tol), float(g_tol)
    P.lambda_init, P.lambda_up, P.lambda_down = float(lambda_init), float(lambda_up), float(lambda_down)
    P.lambda_min, P.lambda_max = float(lambda_min), float(lambda_max)
    P.min_diagonal = float(min_diagonal)
    P.damping = _DAMPING[damping]
    P.covariance = _COV[covariance_estimator]
    P.precision = _PREC[precision]
    return P


def _model_vector(model):
    return np.array([getattr(model, k) for k in _props(model)], dtype=np.float64)


def fit_star_batch(model, cutouts, *, inv_vars=None, origins, inits=None, fixed=None, ctx: Context | None = None,
                   **kw):
    """Many independent fit_star calls in one launch.

    cutouts: list of 2-D arrays (each image[inds]); origins: list of (y1, x1),
    the 1-based image coordinates of each cutout's first pixel; inits: list of
    model parameter vectors (defaults to the model's own values).
    Returns a dict of arrays (params, cov, cost, ..., status).
    """
    fixed = dict(fixed or {})
    ctx = ctx or get_context()
    P = lm_params(model, fixed, **kw)
    n = len(cutouts)
    np_ = len(_props(model))
    dt = np.float32 if all(np.asarray(c).dtype == np.float32 for c in cutouts) else np.float64
    sizes = [np.asarray(c).shape for c in cutouts]
    offs = np.zeros(n, dtype=np.int64)
    tot = 0
    for i, s in enumerate(sizes):
        offs[i] = tot
        tot += s[0] * s[1]
    pix = np.empty(max(tot, 1), dtype=dt)
    for i, c in enumerate(cutouts):
        pix[offs[i]:offs[i] + c.size] = np.asarray(c, dtype=dt).ravel(order="F")
    iv = None
    if inv_vars is not None:
        iv = np.empty(max(tot, 1), dtype=dt)
        for i, c in enumerate(inv_vars):
            if np.asarray(c).shape != sizes[i]:
                raise ArgumentError("`inv_var` must be the same size as `image`")
            iv[offs[i]:offs[i] + sizes[i][0] * sizes[i][1]] = np.asarray(c, dtype=dt).ravel(order="F")
    nyv = np.array([s[0] for s in sizes], dtype=np.int32)
    nxv = np.array([s[1] for s in sizes], dtype=np.int32)
    y1 = np.array([o[0] for o in origins], dtype=np.int32)
    x1 = np.array([o[1] for o in origins], dtype=np.int32)
    init = np.ascontiguousarray(np.stack(inits) if inits is not None else np.tile(_model_vector(model), (n, 1)),
                                dtype=np.float64)
    nf = bin(P.free_mask).count("1")
    out = _lm_outputs(n, np_, nf)
    r = _lm_result_struct(out, lambda a: a.ctypes.data)
    hp = ctx.psf_handle(model)
    et = _abi.CPB_F32 if dt == np.float32 else _abi.CPB_F64
    rc = ctx.lib.cpb_fit_lm_batch(ctx.handle, hp, C.byref(P), n, offs.ctypes.data_as(_abi._i64p),
                                  nyv.ctypes.data_as(_abi._i32p), nxv.ctypes.data_as(_abi._i32p),
                                  y1.ctypes.data_as(_abi._i32p), x1.ctypes.data_as(_abi._i32p),
                                  pix.ctypes.data_as(C.c_void_p),
                                  et, None if iv is None else iv.ctypes.data_as(C.c_void_p),
                                  init.ctypes.data_as(_abi._dp), C.byref(r))
    ctx.raise_for(rc, "cpb_fit_lm_batch")
    out["device_seconds"] = float(r.device_seconds)
    out["names"] = _props(model)
    return out


def _lm_outputs(n, np_, nf):
    return dict(params=np.zeros((n, np_)), cov=np.zeros((n, nf, nf)), cost=np.zeros(n), cost_init=np.zeros(n),
                chisq=np.zeros(n), lambda_final=np.zeros(n), converged=np.zeros(n, np.uint8),
                x_converged=np.zeros(n, np.uint8), f_converged=np.zeros(n, np.uint8),
                g_converged=np.zeros(n, np.uint8), iterations=np.zeros(n, np.int32), status=np.zeros(n, np.int32),
                sigma_final=np.zeros(n))


def _lm_result_struct(out, ptr):
    """LMResultC pointing at the arrays of `out` through ptr(array) (host or device addresses)."""
    r = _abi.LMResultC()
    for f in ("params", "cov", "cost", "cost_init", "chisq", "lambda_final", "sigma_final"):
        setattr(r, f, C.cast(C.c_void_p(ptr(out[f])), _abi._dp) if out.get(f) is not None else None)
    for f in ("converged", "x_converged", "f_converged", "g_converged"):
        setattr(r, f, C.cast(C.c_void_p(ptr(out[f])), _abi._u8p) if out.get(f) is not None else None)
    r.iterations = C.cast(C.c_void_p(ptr(out["iterations"])), _abi._i32p)
    r.status = C.cast(C.c_void_p(ptr(out["status"])), _abi._i32p)
    return r


def fit_star_packed(model, pixels, offsets, ny, nx, y_origin, x_origin, init, *, inv_var=None, fixed=None,
                    ctx: Context | None = None, **kw):
    """Many fit_star calls over cutouts packed in one buffer (the C-ABI layout):
    cutout c is pixels[offsets[c] : offsets[c] + ny[c]*nx[c]], column-major,
    whose first pixel is image pixel (y_origin[c], x_origin[c]) (1-based);
    inv_var (optional) shares the layout; init is (n, np) model parameters.
    float32 pixels are fitted as float32 input, float64 as float64.
    Returns a dict of per-cutout arrays like fit_star_batch."""
    fixed = dict(fixed or {})
    ctx = ctx or get_context()
    P = lm_params(model, fixed, **kw)
    n = len(offsets)
    np_ = len(_props(model))
    nf = bin(P.free_mask).count("1")
    pix = np.ascontiguousarray(pixels)
    dt = np.float32 if pix.dtype == np.float32 else np.float64
    pix = pix.astype(dt, copy=False)
    iv = None if inv_var is None else np.ascontiguousarray(inv_var, dtype=dt)
    if iv is not None and iv.shape != pix.shape:
        raise ArgumentError("`inv_var` must be the same size as `image`")
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    nyv, nxv, y1, x1 = i32(ny), i32(nx), i32(y_origin), i32(x_origin)
    init = np.ascontiguousarray(init, dtype=np.float64).reshape(n, np_)
    out = _lm_outputs(n, np_, nf)
    r = _lm_result_struct(out, lambda a: a.ctypes.data)
    et = _abi.CPB_F32 if dt == np.float32 else _abi.CPB_F64
    rc = ctx.lib.cpb_fit_lm_batch(ctx.handle, ctx.psf_handle(model), C.byref(P), n, offs.ctypes.data_as(_abi._i64p),
                                  nyv.ctypes.data_as(_abi._i32p), nxv.ctypes.data_as(_abi._i32p),
                                  y1.ctypes.data_as(_abi._i32p), x1.ctypes.data_as(_abi._i32p),
                                  pix.ctypes.data_as(C.c_void_p), et,
                                  None if iv is None else iv.ctypes.data_as(C.c_void_p),
                                  init.ctypes.data_as(_abi._dp), C.byref(r))
    ctx.raise_for(rc, "cpb_fit_lm_batch")
    out["device_seconds"] = float(r.device_seconds)
    out["names"] = _props(model)
    return out


def params_matrix(psf, sources):
    """_extract_source_catalog + _build_params_matrix (psf_photometry_single.jl:132-181):
    one row of model parameters per star in getproperties order; y and x from the
    catalogue, flux from it or 1, bkg from it or 0, every other parameter (the
    Gaussian's fwhm) the PSF's own value."""
    names = _props(psf)
    get = (lambda k: sources[k]) if isinstance(sources, dict) else (lambda k: getattr(sources, k))
    has = (lambda k: k in sources) if isinstance(sources, dict) else (lambda k: hasattr(sources, k))
    n = np.asarray(get("y")).size
    default = {"flux": 1.0, "bkg": 0.0}
    cols = []
    for k in names:
        if k in ("y", "x") or (k in default and has(k)):
            v = np.asarray(get(k), dtype=np.float64).ravel()
        else:
            v = np.full(n, default.get(k, float(getattr(psf, k, 0.0))))
        if v.size != n:
            raise ArgumentError(f"source field `{k}` has {v.size} entries, expected {n}")
        cols.append(v)
    return np.ascontiguousarray(np.stack(cols, axis=1)) if n else np.zeros((0, len(names)))


class MultipassOutputs:
    """Caller-owned output arrays of one cpb_multipass_result."""

    def __init__(self, n, np_, ny, nx, residual=True):
        m = max(n, 1)
        self.n, self.np_ = n, np_
        self.params, self.errors = np.zeros((m, np_)), np.zeros((m, np_))
        self.converged, self.valid = np.zeros(m, np.uint8), np.zeros(m, np.uint8)
        self.chisq, self.qfit, self.qfit_expected, self.qfit_z, self.crowding = (np.zeros(m) for _ in range(5))
        self.spread_model, self.spread_model_err = np.zeros(m), np.zeros(m)
        self.n_iter = np.zeros(m, np.int32)
        self.residual = np.zeros((ny, nx), order="F") if residual else None
        r = _abi.MultipassResult()
        dp = lambda a: a.ctypes.data_as(_abi._dp)
        r.params, r.errors = dp(self.params), dp(self.errors)
        r.converged = self.converged.ctypes.data_as(_abi._u8p)
        r.valid = self.valid.ctypes.data_as(_abi._u8p)
        r.chisq, r.qfit, r.qfit_expected = dp(self.chisq), dp(self.qfit), dp(self.qfit_expected)
        r.qfit_z, r.crowding = dp(self.qfit_z), dp(self.crowding)
        r.spread_model, r.spread_model_err = dp(self.spread_model), dp(self.spread_model_err)
        r.n_iter = self.n_iter.ctypes.data_as(_abi._i32p)
        if residual:
            r.residual = dp(self.residual)
        self.c = r

    def result(self, psf, ny, nx) -> MultiPassPhotResult:
        n, names = self.n, _props(psf)
        col = lambda a, k: a[:n, names.index(k)].copy()
        r = self.c
        return MultiPassPhotResult(
            y=col(self.params, "y"), x=col(self.params, "x"), y_err=col(self.errors, "y"),
            x_err=col(self.errors, "x"), flux=col(self.params, "flux"), flux_err=col(self.errors, "flux"),
            bkg=col(self.params, "bkg"), bkg_err=col(self.errors, "bkg"),
            converged=self.converged[:n].astype(bool), valid=self.valid[:n].astype(bool),
            chisq=self.chisq[:n].copy(), qfit=self.qfit[:n].copy(), qfit_expected=self.qfit_expected[:n].copy(),
            qfit_z=self.qfit_z[:n].copy(), crowding=self.crowding[:n].copy(),
            spread_model=self.spread_model[:n].copy(), spread_model_err=self.spread_model_err[:n].copy(),
            n_iter=self.n_iter[:n].astype(np.int64), n_passes=int(r.n_passes), n_failed=int(r.n_failed),
            failure_msgs=[],
            residual=self.residual if self.residual is not None else np.zeros((ny, nx)),
            stats=dict(n_levels=int(r.n_levels), n_fits=int(r.n_fits), device_seconds=float(r.device_seconds),
                       params=self.params[:n].copy()))


def fit_all_stars(image, psf, sources, fit_rad, *, n_passes=3, fixed=None, inv_var=None, spread_model_fwhm=None,
                  ctx: Context | None = None, residual=True, **kw) -> MultiPassPhotResult:
    """CrowdPhot.fit_all_stars on the B200 (psf_photometry_single.jl:267-469): brightness-
    ordered passes of fit_star against the running residual, each pass run as batches of
    stars whose boxes are disjoint (the sequential result).  Keyword arguments other than
    n_passes / fixed / inv_var / spread_model_fwhm go to fit_star (max_iter, x_tol, f_tol,
    g_tol, damping, ...)."""
    fixed = dict(fixed or {})
    ctx = ctx or get_context()
    imgf, ivf, _, et = _image_arrays(image, inv_var, None)
    init = params_matrix(psf, sources)
    P = lm_params(psf, fixed, **kw)
    ny, nx = imgf.shape
    outs = MultipassOutputs(init.shape[0], init.shape[1], ny, nx, residual=residual)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.cpb_fit_all_stars(ctx.handle, ctx.psf_handle(psf), C.byref(P), float(fit_rad), int(n_passes),
                                   spread_fwhm_arg(spread_model_fwhm), vp(imgf), et, ny, nx, vp(ivf), init.shape[0],
                                   init.ctypes.data_as(_abi._dp), C.byref(outs.c))
    ctx.raise_for(rc, "cpb_fit_all_stars")
    return outs.result(psf, ny, nx)


def fit_star(model, image, inds=None, *, fixed=None, inv_var=None, ctx: Context | None = None, **kw):
    """CrowdPhot.PSF.fit_star on the B200 (psf_fitting.jl:229-308) -> (best_model, LMResult).

    inds: ((y_first, y_last), (x_first, x_last)), 1-based inclusive; default the whole image.
    """
    fixed = dict(fixed or {})
    img = np.asarray(image)
    if inv_var is not None and np.asarray(inv_var).shape != img.shape:
        raise ArgumentError("`inv_var` must be the same size as `image`")
    if inds is None:
        inds = ((1, img.shape[0]), (1, img.shape[1]))
    (ya, yb), (xa, xb) = inds
    cut = img[ya - 1:yb, xa - 1:xb]
    ivc = None if inv_var is None else [np.asarray(inv_var)[ya - 1:yb, xa - 1:xb]]
    out = fit_star_batch(model, [cut], inv_vars=ivc, origins=[(ya, xa)], fixed=fixed, ctx=ctx, **kw)
    if out["status"][0] != 0:
        nf = bin(_free_mask(model, fixed)).count("1")
        if ivc is not None:
            iv = ivc[0]
            nvalid = int(np.sum(np.isfinite(iv) & (iv > 0)))
            if not nvalid > nf:
                raise ArgumentError(f"too few valid inv_var pixels ({nvalid}) for {nf} free parameters")
        raise ArgumentError(f"degrees of freedom must be positive; too many free parameters ({nf}) for the number "
                            f"of observations ({cut.size})")
    names = out["names"]
    params = out["params"][0]
    best = replace_params(model, **{k: params[i] for i, k in enumerate(names)})
    free = [i for i, k in enumerate(names) if k not in fixed]
    res = LMResult(minimizer=params[free].copy(), minimum=float(out["cost"][0]), cost_init=float(out["cost_init"][0]),
                   converged=bool(out["converged"][0]), x_converged=bool(out["x_converged"][0]),
                   f_converged=bool(out["f_converged"][0]), g_converged=bool(out["g_converged"][0]),
                   iterations=int(out["iterations"][0]), lambda_final=float(out["lambda_final"][0]),
                   sigma_final=float(out["sigma_final"][0]), cov=out["cov"][0].copy(), chisq=float(out["chisq"][0]))
    return best, res
