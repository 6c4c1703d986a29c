"""spread_model: the band-limited exponential-disk reference kernel and the
diagnostic itself.

The kernel (_exp_disk_kernel_bandlimited, src/photometry/psf_photometry_diagnostics.jl:82-108)
is pinned against the reference's closed form, I(m; v) = exp(-pi^2 m^2 / a)
sqrt(pi / a) Re erf(sqrt(a)/2 + i pi m / sqrt(a)), evaluated here with scipy's
complex erf: both the oracle's restatement (Gauss-Legendre panels) and the
product's host routine (composite Gauss-Legendre, cpb_exp_disk_kernel) must
match it to rounding.  The diagnostic is pinned by the reference's own
known-answer tests (test/photometry/psf_photometry_single.jl:269-321,
test/photometry/psf_photometry_simultaneous.jl:356-383) run on the oracle.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.special as sps

from crowdphot_b200 import CircularGaussianPSF
from crowdphot_b200 import _abi
from crowdphot_b200.simulate import render_sources
from oracle import orc_exp_disk_kernel, orc_fit_all_stars, orc_fit_simultaneous, orc_spread_fwhm

_AMP = (1.99485977e-4, 2.61612679e-3, 1.89726655e-2, 1.00186544e-1, 3.68534484e-1, 5.09490694e-1)
_VAR = (1.20078965e-3, 8.84526493e-3, 3.91463084e-2, 1.39976817e-1, 4.60962500e-1, 1.50159566e0)
CASES = [(fw, h) for fw in (1.0, 2.5, 4.0, 8.0, 20.0) for h in (2, 5, 12, 30)]


def closed_form(fwhm, half):
    re = fwhm / 16 * 1.67834699
    n = 2 * half + 1
    K = np.zeros((n, n))
    for amp, v in zip(_AMP, _VAR):
        a = 2 * np.pi ** 2 * re ** 2 * v
        sa = np.sqrt(a)
        iv = np.array([0.0 if np.pi ** 2 * m * m / a > 690 else
                       np.real(np.exp(-np.pi ** 2 * m * m / a) * np.sqrt(np.pi / a) *
                               sps.erf(sa / 2 + 1j * np.pi * m / sa)) for m in range(-half, half + 1)])
        K += amp * np.outer(iv, iv)
    return K / K.sum()


@pytest.mark.parametrize("fwhm,half", CASES)
def test_oracle_kernel_matches_closed_form(fwhm, half):
    np.testing.assert_allclose(orc_exp_disk_kernel(fwhm, half), closed_form(fwhm, half), rtol=0, atol=1e-13)


@pytest.mark.parametrize("fwhm,half", CASES)
def test_product_kernel_matches_closed_form(fwhm, half):
    """cpb_exp_disk_kernel is host code: it runs without a device."""
    lib = _abi.load_library()
    n = 2 * half + 1
    K = np.zeros(n * n)
    assert lib.cpb_exp_disk_kernel(fwhm, half, K.ctypes.data_as(C.POINTER(C.c_double))) == 0
    np.testing.assert_allclose(K.reshape((n, n), order="F"), closed_form(fwhm, half), rtol=0, atol=1e-13)


def test_product_kernel_argument_errors():
    lib = _abi.load_library()
    K = np.zeros(25)
    p = K.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.cpb_exp_disk_kernel(float("nan"), 2, p) == _abi.CPB_ERR_ARGUMENT
    assert lib.cpb_exp_disk_kernel(0.0, 2, p) == _abi.CPB_ERR_ARGUMENT
    assert lib.cpb_exp_disk_kernel(2.0, -1, p) == _abi.CPB_ERR_ARGUMENT


def test_kernel_invariants():
    """Sum 1, symmetric in both axes, peaked at the centre; a broader disk
    takes more from the centre (the reference's kernel-invariant test)."""
    for fw in (1.5, 2.5, 4.0):
        K = orc_exp_disk_kernel(fw, 5)
        assert K.shape == (11, 11)
        assert abs(K.sum() - 1) < 1e-14
        np.testing.assert_allclose(K, K[::-1, :], atol=1e-15)
        np.testing.assert_allclose(K, K[:, ::-1], atol=1e-15)
        np.testing.assert_allclose(K, K.T, atol=1e-15)
        assert np.unravel_index(np.argmax(K), K.shape) == (5, 5)
    assert orc_exp_disk_kernel(6.0, 5)[5, 5] < orc_exp_disk_kernel(2.0, 5)[5, 5]


def test_spread_fwhm_of_a_gaussian():
    """_spread_fwhm (crowdsource's neff_fwhm) of a well-sampled Gaussian is its FWHM."""
    for fw in (2.5, 4.0, 6.0):
        assert abs(orc_spread_fwhm(CircularGaussianPSF(fwhm=fw), 30.4, 29.7) - fw) < 2e-3 * fw


def _img(shape, y, x, w, flux, bkg=20.0):
    img = np.full(shape, bkg)
    render_sources(img, CircularGaussianPSF(fwhm=w), np.array([y]), np.array([x]), np.array([flux]),
                   model_radius=40)
    return img


FW = 2.5
PSF = CircularGaussianPSF(fwhm=FW)
CAT = dict(y=np.array([30.4]), x=np.array([29.7]), flux=np.array([5000.0]))
KW = dict(n_passes=2, max_iter=100, fixed={"bkg": 20.0, "fwhm": FW})


def test_point_source_is_zero_and_err_needs_weights():
    img = _img((60, 60), 30.4, 29.7, FW, 5000.0)
    r = orc_fit_all_stars(img, PSF, CAT, 8, inv_var=np.full(img.shape, 1 / 20.0), **KW)
    assert r.valid[0]
    assert abs(r.spread_model[0]) < 3e-3
    assert np.isfinite(r.spread_model_err[0]) and r.spread_model_err[0] > 0
    r = orc_fit_all_stars(img, PSF, CAT, 8, **KW)
    assert np.isfinite(r.spread_model[0]) and np.isnan(r.spread_model_err[0])


def test_extended_sources_increase_and_spike_is_negative():
    sm = []
    for w in (2.5, 3.0, 4.0, 6.0):
        img = _img((60, 60), 30.4, 29.7, w, 5000.0)
        sm.append(orc_fit_all_stars(img, PSF, CAT, 8, inv_var=np.full(img.shape, 1 / 20.0), **KW).spread_model[0])
    assert all(s > 5e-4 for s in sm[1:])
    assert sm == sorted(sm)
    spike = np.full((40, 40), 20.0)
    spike[19, 19] += 3000.0
    r = orc_fit_all_stars(spike, PSF, dict(y=np.array([20.0]), x=np.array([20.0]), flux=np.array([3000.0])), 8,
                          inv_var=np.full(spike.shape, 1 / 20.0), **KW)
    assert r.valid[0] and r.spread_model[0] < -1e-3


def test_explicit_disk_width_and_off_switch():
    img = _img((60, 60), 30.4, 29.7, 4.0, 5000.0)
    iv = np.full(img.shape, 1 / 20.0)
    auto = orc_fit_all_stars(img, PSF, CAT, 8, inv_var=iv, **KW)
    big = orc_fit_all_stars(img, PSF, CAT, 8, inv_var=iv, spread_model_fwhm=8.0, **KW)
    assert auto.spread_model[0] > 0 and big.spread_model[0] > auto.spread_model[0]
    for off in (0.0, -1.0, float("nan"), float("inf")):
        r = orc_fit_all_stars(img, PSF, CAT, 8, inv_var=iv, spread_model_fwhm=off, **KW)
        assert np.isnan(r.spread_model[0]) and np.isnan(r.spread_model_err[0])
        assert np.isfinite(r.qfit[0])


def test_simultaneous_matches_sequential():
    """psf_photometry_simultaneous.jl:356-383: three isolated point sources and
    one broadened source, fitted by both paths."""
    img = np.full((90, 90), 20.0)
    pts = [(20.5, 20.5), (20.5, 68.5), (68.5, 20.5)]
    for (yy, xx) in pts:
        render_sources(img, PSF, np.array([yy]), np.array([xx]), np.array([4000.0]), model_radius=40)
    render_sources(img, CircularGaussianPSF(fwhm=5.0), np.array([68.5]), np.array([68.5]), np.array([4000.0]),
                   model_radius=40)
    sub = img - 20.0
    cat = dict(y=np.array([p[0] for p in pts] + [68.5]), x=np.array([p[1] for p in pts] + [68.5]),
               flux=np.full(4, 4000.0))
    iv = np.full(img.shape, 1 / 20.0)
    fixed = {"fwhm": FW, "bkg": 0.0}
    rseq = orc_fit_all_stars(sub, PSF, cat, 7, fixed=fixed, n_passes=3, max_iter=100, inv_var=iv)
    rsim = orc_fit_simultaneous(sub, PSF, cat, 7, fixed=fixed, max_iter=40, inv_var=iv)
    for i in range(3):
        assert rseq.valid[i] and rsim.valid[i]
        assert abs(rseq.spread_model[i]) < 3e-3 and abs(rsim.spread_model[i]) < 3e-3
        assert abs(rseq.spread_model[i] - rsim.spread_model[i]) < 2e-3
    assert rseq.spread_model[3] > 5e-3 and rsim.spread_model[3] > 5e-3
    a, b = rseq.spread_model[3], rsim.spread_model[3]
    assert abs(a - b) <= 0.25 * max(abs(a), abs(b))


def test_simultaneous_disk_width_from_the_fitted_first_star():
    """fit_all_stars_simultaneous sizes the disk after the final bookkeeping, from
    params[row_y, 1], params[row_x, 1] (psf_photometry_simultaneous.jl:1289-1299,
    :1363-1364): the first star's fitted position, not its catalogue one (the
    sequential fit_all_stars takes the catalogue one, psf_photometry_single.jl:324-325)."""
    img = _img((60, 60), 30.4, 29.7, 3.0, 5000.0) - 20.0
    iv = np.full(img.shape, 1 / 20.0)
    cat = dict(y=np.array([30.9]), x=np.array([29.2]), flux=np.array([4000.0]))
    kw = dict(fixed={"fwhm": FW, "bkg": 0.0}, max_iter=40, inv_var=iv)
    auto = orc_fit_simultaneous(img, PSF, cat, 7, **kw)
    assert auto.valid[0] and abs(auto.y[0] - 30.4) < 0.05
    f_fit = orc_spread_fwhm(PSF, auto.y[0], auto.x[0])
    f_cat = orc_spread_fwhm(PSF, 30.9, 29.2)
    assert f_fit != f_cat
    assert orc_fit_simultaneous(img, PSF, cat, 7, spread_model_fwhm=f_fit, **kw).spread_model[0] == \
        auto.spread_model[0]
    assert orc_fit_simultaneous(img, PSF, cat, 7, spread_model_fwhm=f_cat, **kw).spread_model[0] != \
        auto.spread_model[0]
    # a fixed position is the position (the bookkeeping writes the fixed value)
    fx = orc_fit_simultaneous(img, PSF, cat, 7, **dict(kw, fixed={"fwhm": FW, "bkg": 0.0, "y": 30.4}))
    f_fx = orc_spread_fwhm(PSF, 30.4, fx.x[0])
    assert orc_fit_simultaneous(img, PSF, cat, 7, spread_model_fwhm=f_fx,
                                **dict(kw, fixed={"fwhm": FW, "bkg": 0.0, "y": 30.4})).spread_model[0] == \
        fx.spread_model[0]
