"""ctypes binding of oracle/liborc.so (TEST INFRASTRUCTURE ONLY).

orc_fit_simultaneous / orc_fit_star take the same keyword arguments as the
product's fit_all_stars_simultaneous / fit_star and return the same result
types, so a parity test calls both the same way.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "crowdphot.jl_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from crowdphot_b200 import _abi  # noqa: E402  (struct layouts of the shared header)
from crowdphot_b200.photometry import (LMResult, SimOutputs, _catalog, _free_mask, _image_arrays, _props,  # noqa: E402
                                       lm_params, psf_descriptor, sim_params, spread_fwhm_arg)
from crowdphot_b200.psf import ArgumentError, replace_params  # noqa: E402

LIB = os.path.join(_HERE, "liborc.so")
_lib = None
_dp, _i32p, _i64p, _u8p = _abi._dp, _abi._i32p, _abi._i64p, _abi._u8p


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"oracle library missing at {LIB}; run `make -C oracle`")
        lib = C.CDLL(LIB)
        lib.orc_fit_simultaneous.restype = C.c_int
        lib.orc_fit_simultaneous.argtypes = [C.POINTER(_abi.PsfDesc), C.POINTER(_abi.SimParams), C.c_void_p,
                                             C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64,
                                             _dp, _dp, _dp, C.POINTER(_abi.SimResult), C.c_char_p, C.c_int]
        lib.orc_fit_star.restype = C.c_int
        lib.orc_fit_star.argtypes = [C.POINTER(_abi.PsfDesc), C.POINTER(_abi.LMParams), _dp, _dp, C.c_int32,
                                     C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _u8p, _i32p,
                                     C.c_char_p, C.c_int, _dp]
        lib.orc_lm_irls_line.restype = C.c_int
        lib.orc_lm_irls_line.argtypes = [_dp, _dp, C.c_int, C.POINTER(_abi.LMParams), _dp, _dp, _dp, _dp, _i32p]
        lib.orc_estimate_scale.restype = C.c_double
        lib.orc_estimate_scale.argtypes = [C.c_int, C.POINTER(_abi.LMParams), C.c_double, _dp, C.c_int64]
        lib.orc_irls_weight.restype = C.c_double
        lib.orc_irls_weight.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.orc_apply_J.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, _dp, _i32p, _u8p, _dp, _dp]
        lib.orc_apply_JT.argtypes = [C.c_int, C.c_int, C.c_int64, _dp, _i32p, _u8p, _dp, _dp]
        lib.orc_lsqr_stamp.restype = C.c_int
        lib.orc_lsqr_stamp.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, _dp, _i32p, _u8p, _dp, C.c_double,
                                       C.c_int, C.c_double, C.c_double, _dp]
        lib.orc_lsqr_dense.restype = C.c_int
        lib.orc_lsqr_dense.argtypes = [C.c_int64, C.c_int64, _dp, _dp, C.c_double, C.c_int, C.c_double, C.c_double,
                                       _dp]
        lib.orc_lsmr_dense.restype = C.c_int
        lib.orc_lsmr_dense.argtypes = [C.c_int64, C.c_int64, _dp, _dp, C.c_double, C.c_int, C.c_double, C.c_double,
                                       _dp]
        lib.orc_ring_offsets.restype = C.c_int
        lib.orc_ring_offsets.argtypes = [C.c_int, _i32p, _i32p]
        lib.orc_morton2d.restype = C.c_uint64
        lib.orc_morton2d.argtypes = [C.c_int64, C.c_int64]
        lib.orc_bicubic.argtypes = [_dp, C.c_int64, C.c_int64, C.c_int64, _dp, _dp, C.c_double, _dp]
        lib.orc_psf_eval.restype = C.c_int
        lib.orc_psf_eval.argtypes = [C.POINTER(_abi.PsfDesc), C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_int64, _dp, _dp, _dp, _dp]
        lib.orc_fill_stamps.restype = C.c_int
        lib.orc_fill_stamps.argtypes = [C.POINTER(_abi.PsfDesc), C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_int, C.c_int64, C.c_int64, C.c_int64, _i32p,
                                        _i64p, _i64p, _dp, _dp, _u8p, _dp, _dp]
        lib.orc_model_radii_auto_gaussian.restype = C.c_int
        lib.orc_model_radii_auto_gaussian.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int64, _dp,
                                                      C.c_int64, _dp, _i32p]
        lib.orc_exp_disk_kernel.restype = C.c_int
        lib.orc_exp_disk_kernel.argtypes = [C.c_double, C.c_int, _dp]
        lib.orc_spread_fwhm.restype = C.c_double
        lib.orc_spread_fwhm.argtypes = [C.POINTER(_abi.PsfDesc), C.c_double, C.c_double]
        lib.orc_exact_overlap.restype = C.c_double
        lib.orc_exact_overlap.argtypes = [C.c_double, C.c_double, C.c_double]
        lib.orc_aperture_weight.restype = C.c_double
        lib.orc_aperture_weight.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int64]
        lib.orc_unit_curve_of_growth.restype = C.c_int
        lib.orc_unit_curve_of_growth.argtypes = [C.POINTER(_abi.PsfDesc), C.c_double, C.c_int, _dp]
        lib.orc_model_radii_auto.restype = C.c_int
        lib.orc_model_radii_auto.argtypes = [C.POINTER(_abi.PsfDesc), C.c_double, C.c_double, C.c_int, C.c_int,
                                             C.c_int64, _dp, C.c_int64, _dp, _i32p]
        lib.orc_fit_all_stars.restype = C.c_int
        lib.orc_fit_all_stars.argtypes = [C.POINTER(_abi.PsfDesc), C.POINTER(_abi.LMParams), C.c_double, C.c_int,
                                          C.c_double, C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, _dp,
                                          C.POINTER(_abi.MultipassResult), C.c_char_p, C.c_int]
        lib.orc_fit_star_batch.restype = C.c_int
        lib.orc_fit_star_batch.argtypes = [C.POINTER(_abi.PsfDesc), C.POINTER(_abi.LMParams), C.c_int64, _i64p,
                                           _i32p, _i32p, _i32p, _i32p, _dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp,
                                           _dp, _u8p, _i32p, _i32p, C.c_int, _dp]
        _lib = lib
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def orc_fit_simultaneous(image, psf, sources, fit_rad, *, fixed=None, inv_var=None, background=None, debug=False,
                         residual=True, **kw):
    """The oracle's fit_all_stars_simultaneous (same call shape as the product's)."""
    lib = load()
    fixed = dict(fixed or {})
    kw.pop("show_trace", None)
    kw.pop("ctx", None)
    imgf, ivf, bkf, et = _image_arrays(image, inv_var, background)
    y0, x0, f0 = _catalog(sources)
    P = sim_params(psf, fit_rad, fixed, inv_var_given=ivf is not None, **kw)
    ny, nx = imgf.shape
    R = int(np.ceil(fit_rad)) if fit_rad > 0 else 0
    S2 = (2 * R + 1) ** 2
    outs = SimOutputs(y0.size, ny, nx, S2, residual=residual, debug=debug)
    desc, keep = psf_descriptor(psf)
    err = C.create_string_buffer(1024)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = lib.orc_fit_simultaneous(C.byref(desc), C.byref(P), vp(imgf), et, ny, nx, vp(ivf), vp(bkf), y0.size,
                                  y0.ctypes.data_as(_dp), x0.ctypes.data_as(_dp), f0.ctypes.data_as(_dp),
                                  C.byref(outs.c), err, 1024)
    del keep
    if rc != 0:
        raise ArgumentError(err.value.decode())
    return outs.result(ny, nx, S2)


def orc_fit_star(model, image, inds=None, *, fixed=None, inv_var=None, **kw):
    """The oracle's fit_star -> (best_model, LMResult)."""
    lib = load()
    fixed = dict(fixed or {})
    kw.pop("ctx", None)
    P = lm_params(model, fixed, **kw)
    img = np.asarray(image, dtype=np.float64)
    if inds is None:
        inds = ((1, img.shape[0]), (1, img.shape[1]))
    (ya, yb), (xa, xb) = inds
    cut = np.asfortranarray(img[ya - 1:yb, xa - 1:xb])
    ivc = None
    if inv_var is not None:
        if np.asarray(inv_var).shape != img.shape:
            raise ArgumentError("`inv_var` must be the same size as `image`")
        ivc = np.asfortranarray(np.asarray(inv_var, dtype=np.float64)[ya - 1:yb, xa - 1:xb])
    names = _props(model)
    init = np.array([getattr(model, k) for k in names], dtype=np.float64)
    nf = bin(_free_mask(model, fixed)).count("1")
    outp = np.zeros(len(names))
    cov = np.zeros(max(nf * nf, 1))
    sc = [C.c_double() for _ in range(4)]
    flags = np.zeros(4, dtype=np.uint8)
    iters = C.c_int32()
    sigma = C.c_double()
    desc, keep = psf_descriptor(model)
    err = C.create_string_buffer(1024)
    rc = lib.orc_fit_star(C.byref(desc), C.byref(P), cut.ctypes.data_as(_dp),
                          None if ivc is None else ivc.ctypes.data_as(_dp), cut.shape[0], cut.shape[1], ya, xa,
                          init.ctypes.data_as(_dp), outp.ctypes.data_as(_dp), cov.ctypes.data_as(_dp),
                          C.byref(sc[0]), C.byref(sc[1]), C.byref(sc[2]), C.byref(sc[3]),
                          flags.ctypes.data_as(_u8p), C.byref(iters), err, 1024, C.byref(sigma))
    del keep
    if rc != 0:
        raise ArgumentError(err.value.decode())
    best = replace_params(model, **{k: outp[i] for i, k in enumerate(names)})
    free = [i for i, k in enumerate(names) if k not in fixed]
    res = LMResult(minimizer=outp[free].copy(), minimum=sc[0].value, cost_init=sc[1].value, converged=bool(flags[0]),
                   x_converged=bool(flags[1]), f_converged=bool(flags[2]), g_converged=bool(flags[3]),
                   iterations=int(iters.value), lambda_final=sc[3].value, sigma_final=sigma.value,
                   cov=cov[:nf * nf].reshape(nf, nf, order="F").copy(), chisq=sc[2].value)
    return best, res


def orc_apply_J(values, pixels, live, v, npix):
    """values: (n, S2, p) C-order = reference (p, S2, n) column-major; pixels: (n, S2) 1-based."""
    lib = load()
    n, S2, p = values.shape
    y = np.zeros(npix)
    vals, pix, lv, vv = _f64(values), np.ascontiguousarray(pixels, np.int32), np.ascontiguousarray(live, np.uint8), _f64(v)
    lib.orc_apply_J(p, S2, n, npix, vals.ctypes.data_as(_dp), pix.ctypes.data_as(_i32p), lv.ctypes.data_as(_u8p),
                    vv.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
    return y


def orc_apply_JT(values, pixels, live, u):
    lib = load()
    n, S2, p = values.shape
    z = np.zeros(n * p)
    vals, pix, lv, uu = _f64(values), np.ascontiguousarray(pixels, np.int32), np.ascontiguousarray(live, np.uint8), _f64(u)
    lib.orc_apply_JT(p, S2, n, vals.ctypes.data_as(_dp), pix.ctypes.data_as(_i32p), lv.ctypes.data_as(_u8p),
                     uu.ctypes.data_as(_dp), z.ctypes.data_as(_dp))
    return z


def orc_lsqr_stamp(values, pixels, live, rhs, lam, itmax, atol, btol):
    lib = load()
    n, S2, p = values.shape
    x = np.zeros(n * p)
    vals, pix, lv, b = _f64(values), np.ascontiguousarray(pixels, np.int32), np.ascontiguousarray(live, np.uint8), _f64(rhs)
    it = lib.orc_lsqr_stamp(p, S2, n, b.size, vals.ctypes.data_as(_dp), pix.ctypes.data_as(_i32p),
                            lv.ctypes.data_as(_u8p), b.ctypes.data_as(_dp), lam, itmax, atol, btol,
                            x.ctypes.data_as(_dp))
    return x, it


def orc_lsqr_dense(A, b, lam, itmax, atol, btol):
    lib = load()
    m, n = A.shape
    Af = np.asfortranarray(A, dtype=np.float64)
    bb = _f64(b)
    x = np.zeros(n)
    it = lib.orc_lsqr_dense(m, n, Af.ctypes.data_as(_dp), bb.ctypes.data_as(_dp), lam, itmax, atol, btol,
                            x.ctypes.data_as(_dp))
    return x, it


def orc_lsmr_dense(A, b, lam, itmax, atol, btol):
    lib = load()
    m, n = A.shape
    Af = np.asfortranarray(A, dtype=np.float64)
    bb = _f64(b)
    x = np.zeros(n)
    it = lib.orc_lsmr_dense(m, n, Af.ctypes.data_as(_dp), bb.ctypes.data_as(_dp), lam, itmax, atol, btol,
                            x.ctypes.data_as(_dp))
    return x, it


def orc_ring_offsets(R):
    lib = load()
    m = (2 * R + 1) ** 2
    dy = np.zeros(m, np.int32)
    dx = np.zeros(m, np.int32)
    lib.orc_ring_offsets(R, dy.ctypes.data_as(_i32p), dx.ctypes.data_as(_i32p))
    return dy, dx


def orc_morton2d(y, x):
    return int(load().orc_morton2d(int(y), int(x)))


def orc_bicubic(data, y, x, fill=0.0):
    lib = load()
    d = np.asfortranarray(data, dtype=np.float64)
    yy, xx = _f64(np.atleast_1d(y)), _f64(np.atleast_1d(x))
    out = np.zeros(3 * yy.size)
    lib.orc_bicubic(d.ctypes.data_as(_dp), d.shape[0], d.shape[1], yy.size, yy.ctypes.data_as(_dp),
                    xx.ctypes.data_as(_dp), fill, out.ctypes.data_as(_dp))
    return out.reshape(-1, 3)


def orc_psf_eval(psf, y, x, flux, bkg, py, px, grad=True, fwhm=None):
    lib = load()
    desc, keep = psf_descriptor(psf)
    pyy, pxx = _f64(np.atleast_1d(py)), _f64(np.atleast_1d(px))
    f = np.zeros(pyy.size)
    g = np.zeros(3 * pyy.size) if grad else None
    fw = float(fwhm if fwhm is not None else getattr(psf, "fwhm", 0.0))
    rc = lib.orc_psf_eval(C.byref(desc), y, x, flux, bkg, fw, pyy.size, pyy.ctypes.data_as(_dp),
                          pxx.ctypes.data_as(_dp), f.ctypes.data_as(_dp), None if g is None else g.ctypes.data_as(_dp))
    del keep
    if rc != 0:
        raise ArgumentError("bad psf")
    return (f, g.reshape(-1, 3)) if grad else f


def orc_fill_stamps(psf, fixed, R, ny, nx, pixels, anchor_y, anchor_x, theta, w, live, values, colnorm):
    """_fill_stamps! on caller-provided arrays; values (n, S2, p) and colnorm (n, p) updated in place."""
    lib = load()
    desc, keep = psf_descriptor(psf)
    mask = _free_mask(psf, fixed)
    n = pixels.shape[0]
    pix = np.ascontiguousarray(pixels, np.int32)
    ay = np.ascontiguousarray(anchor_y, np.int64)
    ax = np.ascontiguousarray(anchor_x, np.int64)
    th = _f64(theta)
    ww = np.asfortranarray(w, dtype=np.float64)
    lv = np.ascontiguousarray(live, np.uint8)
    assert values.flags["C_CONTIGUOUS"] and values.dtype == np.float64
    assert colnorm.flags["C_CONTIGUOUS"] and colnorm.dtype == np.float64
    rc = lib.orc_fill_stamps(C.byref(desc), mask, float(fixed.get("y", 0.0)), float(fixed.get("x", 0.0)),
                             float(fixed.get("flux", 1.0)), float(fixed.get("bkg", 0.0)),
                             float(fixed.get("fwhm", getattr(psf, "fwhm", 0.0))), R, n, ny, nx,
                             pix.ctypes.data_as(_i32p), ay.ctypes.data_as(_i64p), ax.ctypes.data_as(_i64p),
                             th.ctypes.data_as(_dp), ww.ctypes.data_as(_dp), lv.ctypes.data_as(_u8p),
                             values.ctypes.data_as(_dp), colnorm.ctypes.data_as(_dp))
    del keep
    if rc != 0:
        raise ArgumentError("bad psf")


def orc_exp_disk_kernel(fwhm, half):
    """The oracle's _exp_disk_kernel_bandlimited(fwhm; half) as a (2 half + 1)^2 matrix."""
    n = 2 * int(half) + 1
    K = np.zeros(n * n)
    if load().orc_exp_disk_kernel(float(fwhm), int(half), K.ctypes.data_as(_dp)) != 0:
        raise ArgumentError("invalid exp-disk kernel arguments")
    return K.reshape((n, n), order="F")


def orc_spread_fwhm(psf, y, x):
    """The oracle's _spread_fwhm(psf, y, x)."""
    desc, keep = psf_descriptor(psf)
    v = float(load().orc_spread_fwhm(C.byref(desc), float(y), float(x)))
    del keep
    return v


def orc_exact_overlap(dx, dy, r):
    """Exact area of the unit pixel centred at (dx, dy) inside a circle of radius r at the origin."""
    return float(load().orc_exact_overlap(float(dx), float(dy), float(r)))


def orc_aperture_weight(yc, xc, r, i, j):
    """aperture_weight(CircularAperture(yc, xc, r), i, j, ExactOverlap())."""
    return float(load().orc_aperture_weight(float(yc), float(xc), float(r), int(i), int(j)))


def orc_unit_curve_of_growth(psf, R_cap, fwhm=None):
    lib = load()
    desc, keep = psf_descriptor(psf)
    out = np.zeros(R_cap)
    rc = lib.orc_unit_curve_of_growth(C.byref(desc), float(getattr(psf, "fwhm", 0.0) if fwhm is None else fwhm),
                                      int(R_cap), out.ctypes.data_as(_dp))
    del keep
    if rc != 0:
        raise ArgumentError("bad psf")
    return out


def orc_model_radii_auto(psf, nsigma, R_fit, R_cap, w, flux, fwhm=None):
    lib = load()
    desc, keep = psf_descriptor(psf)
    ww, ff = _f64(w), _f64(flux)
    out = np.zeros(ff.size, np.int32)
    rc = lib.orc_model_radii_auto(C.byref(desc), float(getattr(psf, "fwhm", 0.0) if fwhm is None else fwhm),
                                  float(nsigma), int(R_fit), int(R_cap), ww.size, ww.ctypes.data_as(_dp), ff.size,
                                  ff.ctypes.data_as(_dp), out.ctypes.data_as(_i32p))
    del keep
    if rc != 0:
        raise ArgumentError("no positive weights")
    return out


def orc_model_radii_auto_gaussian(fwhm, nsigma, R_fit, R_cap, w, flux):
    lib = load()
    ww, ff = _f64(w), _f64(flux)
    out = np.zeros(ff.size, np.int32)
    rc = lib.orc_model_radii_auto_gaussian(fwhm, nsigma, R_fit, R_cap, ww.size, ww.ctypes.data_as(_dp), ff.size,
                                           ff.ctypes.data_as(_dp), out.ctypes.data_as(_i32p))
    if rc != 0:
        raise ArgumentError("no positive weights")
    return out


def orc_fit_star_packed(model, pix, offsets, ny, nx, y1, x1, init, *, inv_var=None, fixed=None, threads=0, **kw):
    """The oracle's fit_star over many packed cutouts (same layout as
    crowdphot_b200.fit_star_packed), spread over `threads` host threads
    (0 = all).  Returns (dict of per-cutout arrays, threads used)."""
    lib = load()
    fixed = dict(fixed or {})
    P = lm_params(model, fixed, **kw)
    n = len(offsets)
    names = _props(model)
    np_ = len(names)
    nf = bin(_free_mask(model, fixed)).count("1")
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    pix, init = f64(pix), f64(init)
    iv = None if inv_var is None else f64(inv_var)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    ny, nx, y1, x1 = i32(ny), i32(nx), i32(y1), i32(x1)
    out = dict(params=np.zeros((n, np_)), cov=np.zeros((n, nf, nf)), scal=np.zeros((n, 4)),
               flags=np.zeros((n, 4), np.uint8), iterations=np.zeros(n, np.int32), status=np.zeros(n, np.int32),
               sigma_final=np.zeros(n))
    desc, keep = psf_descriptor(model)
    used = lib.orc_fit_star_batch(C.byref(desc), C.byref(P), n, offsets.ctypes.data_as(_i64p),
                                  ny.ctypes.data_as(_i32p), nx.ctypes.data_as(_i32p), y1.ctypes.data_as(_i32p),
                                  x1.ctypes.data_as(_i32p), pix.ctypes.data_as(_dp),
                                  None if iv is None else iv.ctypes.data_as(_dp), init.ctypes.data_as(_dp), np_, nf,
                                  out["params"].ctypes.data_as(_dp), out["cov"].ctypes.data_as(_dp),
                                  out["scal"].ctypes.data_as(_dp), out["flags"].ctypes.data_as(_u8p),
                                  out["iterations"].ctypes.data_as(_i32p), out["status"].ctypes.data_as(_i32p),
                                  int(threads), out["sigma_final"].ctypes.data_as(_dp))
    del keep
    if used < 0:
        raise ArgumentError("invalid PSF descriptor")
    sc, fl = out.pop("scal"), out.pop("flags")
    out.update(cost=sc[:, 0].copy(), cost_init=sc[:, 1].copy(), chisq=sc[:, 2].copy(), lambda_final=sc[:, 3].copy(),
               converged=fl[:, 0].copy(), x_converged=fl[:, 1].copy(), f_converged=fl[:, 2].copy(),
               g_converged=fl[:, 3].copy(), names=names)
    return out, used


def orc_fit_all_stars(image, psf, sources, fit_rad, *, n_passes=3, fixed=None, inv_var=None, residual=True,
                      spread_model_fwhm=None, **kw):
    """The oracle's fit_all_stars (same call shape as the product's)."""
    from crowdphot_b200.photometry import MultipassOutputs, params_matrix
    lib = load()
    fixed = dict(fixed or {})
    kw.pop("ctx", None)
    imgf, ivf, _, et = _image_arrays(image, inv_var, None)
    init = params_matrix(psf, sources)
    P = lm_params(psf, fixed, **kw)
    ny, nx = imgf.shape
    outs = MultipassOutputs(init.shape[0], init.shape[1], ny, nx, residual=residual)
    desc, keep = psf_descriptor(psf)
    err = C.create_string_buffer(1024)
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = lib.orc_fit_all_stars(C.byref(desc), C.byref(P), float(fit_rad), int(n_passes),
                               spread_fwhm_arg(spread_model_fwhm), vp(imgf), et, ny, nx, vp(ivf),
                               init.shape[0], init.ctypes.data_as(_dp), C.byref(outs.c), err, 1024)
    del keep
    if rc != 0:
        raise ArgumentError(err.value.decode())
    return outs.result(psf, ny, nx)


def orc_lm_irls_line(xs, ys, x0=(0.0, 0.0), **kw):
    """lm_irls on the reference's straight-line test problem -> (x, lambda_final, sigma_final, iterations).
    Keyword arguments are lm_irls's (reweight, scale_estimator, weight_reset_tol, tolerances, ...)."""
    from crowdphot_b200 import CircularGaussianPSF
    lib = load()
    P = lm_params(CircularGaussianPSF(fwhm=1.0), {}, **kw)
    xs, ys, x0 = _f64(xs), _f64(ys), _f64(x0)
    xo, lam, sig, it = np.zeros(2), C.c_double(), C.c_double(), C.c_int32()
    rc = lib.orc_lm_irls_line(xs.ctypes.data_as(_dp), ys.ctypes.data_as(_dp), xs.size, C.byref(P),
                              x0.ctypes.data_as(_dp), xo.ctypes.data_as(_dp), C.byref(lam), C.byref(sig), C.byref(it))
    if rc != 0:
        raise ArgumentError("degrees of freedom must be positive")
    return xo, lam.value, sig.value, it.value


def orc_estimate_scale(estimator, r):
    """estimate_scale(estimator, r) for MADScale / FixedScale / MScale."""
    from crowdphot_b200 import CircularGaussianPSF
    P = lm_params(CircularGaussianPSF(fwhm=1.0), {}, reweight=None, scale_estimator=estimator)
    rr = _f64(r)
    return float(load().orc_estimate_scale(P.scale_estimator, C.byref(P), P.scale_value, rr.ctypes.data_as(_dp),
                                           rr.size))


def orc_irls_weight(loss, r):
    """weight(loss, r) for L2DistLoss / HuberLoss / TukeyLoss / LogitDistLoss."""
    from crowdphot_b200 import CircularGaussianPSF
    P = lm_params(CircularGaussianPSF(fwhm=1.0), {}, reweight=loss)
    return float(load().orc_irls_weight(P.reweight, P.loss_param, float(r)))
