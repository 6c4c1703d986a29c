"""fit_all_stars on the device (cpb_fit_all_stars: brightness-ordered passes run
as batches of stars with disjoint boxes) against the oracle's one-star-at-a-time
restatement, on the same seeded inputs.  The batches reproduce the sequential
order, so the gates are tight: validity, convergence and iteration counts
equal; parameters and errors within 1e-8 relative (FP64 rounding of the model
renders); diagnostics within 1e-6."""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF
from crowdphot_b200.simulate import crowded_field, moffat_epsf
from oracle import orc_fit_all_stars
from test_oracle_multipass import field

pytestmark = pytest.mark.gpu


def compare(g, o, rtol=1e-8):
    assert g.n_passes == o.n_passes and g.n_failed == o.n_failed
    assert np.array_equal(g.valid, o.valid)
    assert np.array_equal(g.converged, o.converged)
    assert (g.n_iter == o.n_iter).mean() >= 0.99
    ok = g.valid & (g.n_iter == o.n_iter)
    for k in ("y", "x"):
        np.testing.assert_allclose(getattr(g, k)[ok], getattr(o, k)[ok], rtol=0, atol=1e-7)
    for k in ("flux", "bkg", "flux_err", "y_err", "chisq"):
        np.testing.assert_allclose(getattr(g, k)[ok], getattr(o, k)[ok], rtol=rtol, atol=1e-10)
    for k in ("qfit", "qfit_expected", "qfit_z", "crowding"):
        np.testing.assert_allclose(getattr(g, k)[ok], getattr(o, k)[ok], rtol=1e-6, atol=1e-10)


def test_crowded_epsf_three_passes():
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(192, 192, 420, seed=3001, psf=psf, dtype=np.float32)
    data = (img - bkg).astype(np.float32)
    kw = dict(n_passes=3, fixed={"bkg": 0.0}, inv_var=iv, max_iter=100)
    g = cpb.fit_all_stars(data, psf, init, 8, **kw)
    o = orc_fit_all_stars(data, psf, init, 8, **kw)
    print(f"batches over 3 passes: {g.stats['n_levels']}, fits {g.stats['n_fits']}, valid {g.valid.sum()}/420")
    assert g.stats["n_levels"] < g.stats["n_fits"] / 4  # batches really hold many stars
    compare(g, o)
    np.testing.assert_allclose(g.residual, o.residual, rtol=0, atol=1e-6 * (1 + np.abs(o.residual).max()))


def test_gaussian_noiseless_and_edge_cases():
    psf = CircularGaussianPSF(fwhm=2.0)
    img, src = field((128, 128), 5, 1)
    g = cpb.fit_all_stars(img, psf, src, 5, n_passes=3, max_iter=100, fixed={"bkg": 20.0})
    o = orc_fit_all_stars(img, psf, src, 5, n_passes=3, max_iter=100, fixed={"bkg": 20.0})
    compare(g, o)
    np.testing.assert_allclose(g.y, src["y"], atol=0.01)
    # a star rejected between passes (non-positive flux) and an edge star, free bkg and fwhm
    img, src = field((64, 64), 5, 4, flux=(400.0, 700.0), min_sep=10)
    bad = dict(y=np.r_[src["y"], 50.0, 1.0], x=np.r_[src["x"], 50.0, 30.0], flux=np.r_[src["flux"], -100.0, 300.0])
    g = cpb.fit_all_stars(img, psf, bad, 5, n_passes=2, max_iter=100)
    o = orc_fit_all_stars(img, psf, bad, 5, n_passes=2, max_iter=100)
    assert not g.valid[5]
    compare(g, o)
    r = cpb.fit_all_stars(img, psf, dict(y=[], x=[], flux=[]), 5)
    assert r.flux.size == 0
    with pytest.raises(ArgumentError, match="n_passes"):
        cpb.fit_all_stars(img, psf, src, 5, n_passes=0)
