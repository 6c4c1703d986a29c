"""The oracle's fit_all_stars (psf_photometry_single.jl:267-469) against the
reference's own RNG-independent expectations (test/photometry/psf_photometry_single.jl:
105-266): noiseless recovery of separated stars, fixed background / positions,
qfit_expected with weights, rejection of a non-positive flux between passes,
and the result layout."""
import numpy as np
import pytest

from crowdphot_b200 import CircularGaussianPSF
from crowdphot_b200.simulate import render_sources
from oracle import orc_fit_all_stars

TRUTH = dict(fwhm=2.0)


def field(shape, n, seed, flux=(600.0, 900.0), min_sep=7.0, border=8, bkg=20.0):
    rng = np.random.default_rng(seed)
    ys, xs = [], []
    for _ in range(100000):
        if len(ys) == n:
            break
        y = rng.uniform(border, shape[0] - border)
        x = rng.uniform(border, shape[1] - border)
        if all((y - a) ** 2 + (x - b) ** 2 >= min_sep ** 2 for a, b in zip(ys, xs)):
            ys.append(y)
            xs.append(x)
    assert len(ys) == n, "placement failed"
    f = rng.uniform(*flux, n)
    img = np.full(shape, bkg)
    render_sources(img, CircularGaussianPSF(fwhm=2.0), np.array(ys), np.array(xs), f, model_radius=30)
    return img, dict(y=np.array(ys), x=np.array(xs), flux=f)


def test_noiseless_recovery_three_passes():
    img, src = field((128, 128), 5, 1)
    psf = CircularGaussianPSF(fwhm=2.0)
    r = orc_fit_all_stars(img, psf, src, 5, n_passes=3, max_iter=100, fixed={"bkg": 20.0})
    assert r.n_passes == 3 and r.n_failed == 0
    assert r.valid.all() and r.converged.all()
    np.testing.assert_allclose(r.flux, src["flux"], rtol=0.10)
    np.testing.assert_allclose(r.y, src["y"], atol=0.01)
    np.testing.assert_allclose(r.x, src["x"], atol=0.01)
    assert np.all(np.isfinite(r.qfit)) and np.all(r.qfit >= 0)
    assert np.all(np.isnan(r.qfit_expected)) and np.all(np.isnan(r.qfit_z))
    assert np.all(np.isfinite(r.crowding)) and np.all(r.crowding >= 0)
    assert r.residual.shape == img.shape


def test_single_pass_with_weights_and_fixed_parameters():
    img, src = field((128, 128), 5, 2, min_sep=10, border=10)
    psf = CircularGaussianPSF(fwhm=2.0)
    r = orc_fit_all_stars(img, psf, src, 5, n_passes=1, max_iter=100, inv_var=np.ones(img.shape))
    assert r.valid.all() and r.converged.all()
    assert np.all(np.isfinite(r.qfit_expected)) and np.all(r.qfit_expected > 0) and np.all(np.isfinite(r.qfit_z))
    img, src = field((64, 64), 5, 3, flux=(500.0, 800.0), min_sep=10)
    r = orc_fit_all_stars(img, psf, src, 5, fixed={"bkg": 20.0}, n_passes=1, max_iter=100)
    np.testing.assert_allclose(r.bkg, 20.0)
    assert np.all(r.bkg_err == 0)
    np.testing.assert_allclose(r.flux, src["flux"], rtol=0.02)
    r = orc_fit_all_stars(img, psf, src, 5, fixed={"x": 32.0, "y": 32.0}, n_passes=1, max_iter=100)
    np.testing.assert_allclose(r.x, 32.0)
    np.testing.assert_allclose(r.y, 32.0)
    assert np.all(r.x_err == 0) and np.all(r.y_err == 0)


def test_invalid_flux_rejected_between_passes_and_edge_star():
    img, src = field((64, 64), 5, 4, flux=(400.0, 700.0), min_sep=10)
    psf = CircularGaussianPSF(fwhm=2.0)
    bad = dict(y=np.r_[src["y"], 50.0], x=np.r_[src["x"], 50.0], flux=np.r_[src["flux"], -100.0])
    r = orc_fit_all_stars(img, psf, bad, 5, n_passes=2, max_iter=100)
    assert r.valid.sum() == 5 and not r.valid[5]
    img = np.full((64, 64), 20.0)
    render_sources(img, psf, np.array([1.5, 32.2]), np.array([32.0, 31.8]), np.array([520.0, 580.0]), model_radius=30)
    r = orc_fit_all_stars(img, psf, dict(y=[1.0, 32.0], x=[32.0, 32.0], flux=[500.0, 500.0]), 5, n_passes=1,
                          max_iter=50)
    assert r.valid[1]
    with pytest.raises(Exception, match="n_passes"):
        orc_fit_all_stars(img, psf, dict(y=[32.0], x=[32.0], flux=[5.0]), 5, n_passes=0)
