"""fit_star with IRLS reweighting on the device (k_lm_irls) against the oracle's
lm_irls, cutout by cutout, on the same seeded inputs: every loss (L2DistLoss,
HuberLoss, TukeyLoss, LogitDistLoss) and scale estimator (the default, MADScale, FixedScale,
MScale), with and without inv_var, for the ePSF, a four-node gridded PSF and
the Gaussian (free FWHM).  The weights are recomputed from residuals divided by
a median-based scale, so the device's rounding (fused multiply-adds, warp
reductions) can move a trajectory by a step; the gates allow 3 % of the cutouts
a different iteration count and compare the rest tightly."""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import (ArgumentError, CircularGaussianPSF, FixedScale, HuberLoss, L2DistLoss, LogitDistLoss,
                            MADScale, MScale, TukeyLoss)
from crowdphot_b200.simulate import lm_cutouts, moffat_epsf
from oracle import orc_fit_star
from oracle.ffi import orc_fit_star_packed

pytestmark = pytest.mark.gpu


def compare(g, o, np_pos=2):
    assert np.array_equal(g["status"], o["status"])
    ok = g["status"] == 0
    same = ok & (g["iterations"] == o["iterations"])
    assert same.sum() >= 0.97 * ok.sum(), f"{ok.sum() - same.sum()} of {ok.sum()} cutouts took other paths"
    assert np.array_equal(g["converged"][same], o["converged"][same])
    assert np.max(np.abs(g["params"][same, :np_pos] - o["params"][same, :np_pos])) < 1e-6
    np.testing.assert_allclose(g["params"][same, np_pos:], o["params"][same, np_pos:], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(g["sigma_final"][same], o["sigma_final"][same], rtol=1e-7, equal_nan=True)
    np.testing.assert_allclose(g["chisq"][same], o["chisq"][same], rtol=1e-6)
    np.testing.assert_allclose(g["lambda_final"][same], o["lambda_final"][same], rtol=1e-9)
    np.testing.assert_allclose(g["cov"][same], o["cov"][same], rtol=1e-5, atol=1e-12)
    return same


CASES = [(HuberLoss(1.0), None), (TukeyLoss(), None), (L2DistLoss(), MADScale()), (HuberLoss(1.5), MScale()),
         (TukeyLoss(4.0), FixedScale(1.3)), (LogitDistLoss(), MADScale())]


@pytest.mark.parametrize("loss,scale", CASES)
@pytest.mark.parametrize("weights", [True, False])
def test_epsf_cutouts_match_oracle(loss, scale, weights):
    psf = moffat_epsf()
    d = lm_cutouts(600, seed=77, dtype=np.float64)
    # a few cosmic-ray hits, the case IRLS is for
    rng = np.random.default_rng(5)
    hit = rng.integers(0, d["pix"].size, 400)
    d["pix"][hit] += rng.uniform(200, 2000, hit.size)
    args = (d["pix"], d["offsets"], d["ny"], d["nx"], d["y1"], d["x1"], d["init"])
    kw = dict(fixed={"bkg": 0.0}, reweight=loss, scale_estimator=scale, inv_var=d["inv_var"] if weights else None)
    g = cpb.fit_star_packed(psf, *args, **kw)
    o, _ = orc_fit_star_packed(psf, *args, threads=0, **kw)
    same = compare(g, o)
    assert np.all(np.isfinite(g["sigma_final"][same]) | np.isnan(o["sigma_final"][same]))


def test_gaussian_and_four_node_gridded():
    from test_gpu_sim import four_node_epsf
    # Gaussian with free FWHM and background, noiseless parity and outliers (psf_fitting_tests.jl:255-317)
    truth = CircularGaussianPSF(x=15.0, y=15.0, fwhm=4.0, flux=200.0, bkg=1.0)
    i = np.arange(1, 31, dtype=float)[:, None]
    j = np.arange(1, 31, dtype=float)[None, :]
    base = truth.evaluate(i, j)
    init = CircularGaussianPSF(x=15.5, y=14.5, fwhm=3.5, flux=180.0, bkg=1.5)
    for seed in range(6):
        img = base + 0.5 * np.random.default_rng(seed).standard_normal(base.shape)
        for (a, b) in [(5, 5), (25, 6), (8, 24), (15, 28), (22, 12)]:
            img[a - 1, b - 1] += 10.0
        for loss in (HuberLoss(1.0), TukeyLoss(), MScale()):
            kw = dict(reweight=loss, max_iter=500) if not isinstance(loss, MScale) else \
                dict(reweight=HuberLoss(1.0), scale_estimator=loss, max_iter=500)
            bg, rg = cpb.fit_star(init, img, **kw)
            bo, ro = orc_fit_star(init, img, **kw)
            assert rg.iterations == ro.iterations and rg.converged == ro.converged
            assert abs(bg.flux / bo.flux - 1) < 1e-8 and abs(bg.fwhm - bo.fwhm) < 1e-8
            assert rg.sigma_final == pytest.approx(ro.sigma_final, rel=1e-8)
            assert rg.chisq == pytest.approx(ro.chisq, rel=1e-8)
    # four-node gridded PSF (the generic corner blend)
    g4 = four_node_epsf()
    d = lm_cutouts(200, seed=78, psf=moffat_epsf(fwhm=2.8, size=121), dtype=np.float64)
    y1 = 20 + (d["y1"] % 80)
    x1 = 20 + (d["x1"] % 80)
    shift_y, shift_x = (y1 - d["y1"]).astype(float), (x1 - d["x1"]).astype(float)
    init = d["init"].copy()
    init[:, 0] += shift_y
    init[:, 1] += shift_x
    args = (d["pix"], d["offsets"], d["ny"], d["nx"], y1, x1, init)
    kw = dict(fixed={"bkg": 0.0}, reweight=TukeyLoss(), inv_var=d["inv_var"])
    compare(cpb.fit_star_packed(g4, *args, **kw), orc_fit_star_packed(g4, *args, threads=0, **kw)[0])


def test_irls_argument_errors_and_plain_sigma():
    psf = moffat_epsf()
    d = lm_cutouts(4, seed=79, dtype=np.float64)
    args = (d["pix"], d["offsets"], d["ny"], d["nx"], d["y1"], d["x1"], d["init"])
    with pytest.raises(ArgumentError, match="non-negative"):
        cpb.fit_star_packed(psf, *args, reweight=HuberLoss(1.0), weight_reset_tol=-0.5)
    with pytest.raises(ArgumentError, match="strictly positive"):
        cpb.fit_star_packed(psf, *args, reweight=HuberLoss(0.0))
    g = cpb.fit_star_packed(psf, *args, fixed={"bkg": 0.0})
    assert np.all(np.isnan(g["sigma_final"]))
