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
    for k in ("qfit", "qfit_expected", "qfit_z", "crowding", "spread_model_err"):
        np.testing.assert_allclose(getattr(g, k)[ok], getattr(o, k)[ok], rtol=1e-6, atol=1e-10)
    # spread_model is a difference of two ratios near 1 (about 0 for a point source)
    np.testing.assert_allclose(g.spread_model[ok], o.spread_model[ok], rtol=1e-6, atol=1e-8)
    assert np.array_equal(np.isnan(g.spread_model), np.isnan(o.spread_model))


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


def test_spread_model_known_answers_and_wide_boxes():
    """The reference's spread_model expectations (test/photometry/psf_photometry_single.jl:
    269-321) on the device, each against the oracle; a 30 px fit radius (model stamps
    of 63 x 63 per warp, fewer warps per block) and the off switch."""
    from test_oracle_spread import CAT, FW, KW, PSF, _img
    iv = np.full((60, 60), 1 / 20.0)
    sm = []
    for w in (2.5, 3.0, 4.0, 6.0):
        img = _img((60, 60), 30.4, 29.7, w, 5000.0)
        g = cpb.fit_all_stars(img, PSF, CAT, 8, inv_var=iv, **KW)
        compare(g, orc_fit_all_stars(img, PSF, CAT, 8, inv_var=iv, **KW))
        sm.append(g.spread_model[0])
    assert abs(sm[0]) < 3e-3 and all(s > 5e-4 for s in sm[1:]) and sm == sorted(sm)
    img = _img((60, 60), 30.4, 29.7, 4.0, 5000.0)
    g = cpb.fit_all_stars(img, PSF, CAT, 8, inv_var=iv, spread_model_fwhm=8.0, **KW)
    compare(g, orc_fit_all_stars(img, PSF, CAT, 8, inv_var=iv, spread_model_fwhm=8.0, **KW))
    assert g.spread_model[0] > sm[2]
    g = cpb.fit_all_stars(img, PSF, CAT, 8, inv_var=iv, spread_model_fwhm=0.0, **KW)
    assert np.isnan(g.spread_model[0]) and np.isnan(g.spread_model_err[0]) and np.isfinite(g.qfit[0])
    g = cpb.fit_all_stars(img, PSF, CAT, 8, **KW)
    assert np.isfinite(g.spread_model[0]) and np.isnan(g.spread_model_err[0])
    big, src = field((160, 160), 4, 5, min_sep=40, border=35)
    kw = dict(n_passes=2, max_iter=100, fixed={"bkg": 20.0}, inv_var=np.ones(big.shape))
    g = cpb.fit_all_stars(big, CircularGaussianPSF(fwhm=2.0), src, 30, **kw)
    o = orc_fit_all_stars(big, CircularGaussianPSF(fwhm=2.0), src, 30, **kw)
    assert np.all(np.isfinite(g.spread_model[g.valid]))
    compare(g, o)


def test_batch_level_path_irls_and_four_node_psf():
    """The batch-by-batch path (fit_star launches per batch) serves what the
    dependency-driven launch does not: IRLS reweighting and multi-node gridded
    PSFs.  Both against the oracle."""
    from crowdphot_b200 import HuberLoss
    from test_gpu_sim import four_node_epsf
    psf = CircularGaussianPSF(fwhm=2.0)
    img, src = field((96, 96), 12, 6, min_sep=6)
    kw = dict(n_passes=2, max_iter=100, fixed={"bkg": 20.0}, reweight=HuberLoss(1.0))
    compare(cpb.fit_all_stars(img, psf, src, 5, **kw), orc_fit_all_stars(img, psf, src, 5, **kw))
    g4 = four_node_epsf()
    from oracle import orc_psf_eval
    rng = np.random.default_rng(11)
    ys, xs = rng.uniform(12, 118, 40), rng.uniform(12, 118, 40)
    fl = rng.uniform(500, 5000, 40)
    img = np.zeros((128, 128))
    yy, xx = np.meshgrid(np.arange(1, 129), np.arange(1, 129), indexing="ij")
    for y, x, f in zip(ys, xs, fl):
        img += orc_psf_eval(g4, y, x, f, 0.0, yy.ravel().astype(float), xx.ravel().astype(float),
                            grad=False).reshape(img.shape)
    img += rng.normal(0, 1.0, img.shape)
    iv = np.ones(img.shape)
    cat = dict(y=ys + rng.normal(0, 0.2, 40), x=xs + rng.normal(0, 0.2, 40), flux=fl)
    kw = dict(n_passes=2, max_iter=60, fixed={"bkg": 0.0}, inv_var=iv)
    compare(cpb.fit_all_stars(img, g4, cat, 6, **kw), orc_fit_all_stars(img, g4, cat, 6, **kw))


def test_bounded_wait_runs_out_and_the_context_stays_usable():
    """Every device-side wait of the dependency-driven pass kernel is bounded.  The
    host holds the brightest star of the first pass back from the ready queue
    (cpb_ctx_inject_fault; no GPU fault), so the stars behind it never become ready:
    with a short wait limit the call returns CPB_ERR_TIMEOUT (TimeoutError) with the
    reason, and the next call on the same context gives the same result as before."""
    from crowdphot_b200 import _abi
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(128, 128, 160, seed=3005, psf=psf, dtype=np.float32)
    data = (img - bkg).astype(np.float32)
    kw = dict(n_passes=2, fixed={"bkg": 0.0}, inv_var=iv, max_iter=100)
    ctx = cpb.get_context(0)
    before = cpb.fit_all_stars(data, psf, init, 8, ctx=ctx, **kw)
    assert before.valid.sum() > 100
    try:
        ctx.set_wait_limit(20_000)  # about a few ms of polling per wait
        ctx.inject_fault(_abi.CPB_FAULT_HOLD_READY_STAR)
        with pytest.raises(TimeoutError, match="stalled waiting for ready stars"):
            cpb.fit_all_stars(data, psf, init, 8, ctx=ctx, **kw)
    finally:
        ctx.set_wait_limit(0)
        ctx.inject_fault(_abi.CPB_FAULT_NONE)
    after = cpb.fit_all_stars(data, psf, init, 8, ctx=ctx, **kw)
    for k in ("y", "x", "flux", "flux_err", "valid", "converged", "n_iter"):
        assert np.array_equal(getattr(after, k), getattr(before, k)), k
    with pytest.raises(ArgumentError, match="unknown fault"):
        ctx.inject_fault(7)
