"""End-to-end oracle fits against the reference test suite's known answers.

Restates test/photometry/psf_photometry_simultaneous.jl:219-253 (noiseless
isolated stars recover the truth), :294-334 (contract errors, empty input,
failure paths), :336-354 (qfit definition), :407-453 (per-star freezing),
:466-497 (_model_radii) and test/psf/psf_fitting_tests.jl / psf_fit_parity_tests.jl
(fit_star noiseless recovery, 4-corner gridded model) with numpy RNGs.
"""
import numpy as np
import pytest

from crowdphot_b200 import ArgumentError, CircularGaussianPSF, GriddedPSFModel, ImagePSF
from crowdphot_b200.simulate import render_sources, simulate_sources, add_noise
from oracle import orc_fit_simultaneous, orc_fit_star, orc_model_radii_auto_gaussian


def gaussian_node_psf(fwhm=2.0, half=7):
    g = CircularGaussianPSF(fwhm=fwhm)
    off = np.arange(-half, half + 1, dtype=float)
    data = g.evaluate(off[:, None], off[None, :])
    node = ImagePSF(data, oversampling=1, normalize=True)
    return GriddedPSFModel([node], [0.0], [0.0])


def isolated_field(psf, seed=42, shape=(128, 128), n=5):
    rng = np.random.default_rng(seed)
    src = simulate_sources(shape, n, rng=rng, flux=(600.0, 900.0), min_separation=15, border=10)
    img = np.zeros(shape)
    render_sources(img, psf, src["y"], src["x"], src["flux"], model_radius=5)
    return img, src


@pytest.mark.parametrize("solver", ["lsqr", "lsmr"])
@pytest.mark.parametrize("kind", ["gaussian", "gridded"])
def test_isolated_noiseless_recovers_truth(kind, solver):
    psf = CircularGaussianPSF(fwhm=2.0) if kind == "gaussian" else gaussian_node_psf()
    fixed = {"fwhm": 2.0, "bkg": 0.0} if kind == "gaussian" else {"bkg": 0.0}
    img, src = isolated_field(psf)
    cat = dict(y=src["y"], x=src["x"], flux=np.full(5, 400.0))
    r = orc_fit_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=40, inner_iterations=10, x_tol=1e-8,
                             model_rad=5, solver=solver)
    assert r.valid.all()
    np.testing.assert_allclose(r.flux, src["flux"], rtol=1e-10)
    np.testing.assert_allclose(r.y, src["y"], atol=1e-10)
    np.testing.assert_allclose(r.x, src["x"], atol=1e-10)
    assert np.all(r.flux_err > 0) and np.all(r.y_err > 0)


def test_free_set_contract_errors():
    psf = CircularGaussianPSF(fwhm=2.0)
    img = np.zeros((64, 64))
    cat = dict(y=[32.0], x=[32.0], flux=[500.0])
    with pytest.raises(ArgumentError, match="fits only"):
        orc_fit_simultaneous(img, psf, cat, 5, model_rad=5)
    with pytest.raises(ArgumentError, match="LevenbergDamping"):
        orc_fit_simultaneous(img, psf, cat, 5, fixed={"fwhm": 2.0, "bkg": 0.0}, damping="levenberg", model_rad=5)
    with pytest.raises(ArgumentError, match="solver"):
        orc_fit_simultaneous(img, psf, cat, 5, fixed={"fwhm": 2.0, "bkg": 0.0}, solver="foo", model_rad=5)
    for kw, msg in [(dict(max_iter=0), "max_iter"), (dict(inner_iterations=0), "inner_iterations"),
                    (dict(linear_tol=0.0), "linear_tol"), (dict(max_trials=0), "max_trials"),
                    (dict(model_rad=-1.0), "model_rad"), (dict(model_rad_max=1.0), "model_rad_max"),
                    (dict(model_rad_nsigma=0.0), "nsigma")]:
        kw.setdefault("model_rad", 5)
        with pytest.raises(ArgumentError, match=msg):
            orc_fit_simultaneous(img, psf, cat, 5, fixed={"fwhm": 2.0, "bkg": 0.0}, **kw)


def test_empty_input_and_failure_paths():
    psf = CircularGaussianPSF(fwhm=2.0)
    fixed = {"fwhm": 2.0, "bkg": 0.0}
    r = orc_fit_simultaneous(np.zeros((16, 16)), psf, dict(y=[], x=[], flux=[]), 5, fixed=fixed)
    assert r.flux.size == 0 and r.n_passes == 0
    bad = np.zeros((32, 32))
    bad[4, 4] = np.nan
    with pytest.raises(ArgumentError, match="non-finite"):
        orc_fit_simultaneous(bad, psf, dict(y=[16.0], x=[16.0], flux=[100.0]), 5, fixed=fixed, model_rad=5)
    iv = np.ones((32, 32))
    iv[9:22, 9:22] = 0
    r = orc_fit_simultaneous(np.zeros((32, 32)), psf, dict(y=[16.0], x=[16.0], flux=[100.0]), 5, fixed=fixed,
                             inv_var=iv)
    assert r.n_failed == 1 and not r.valid[0]
    with pytest.raises(ArgumentError, match="requires inv_var"):
        orc_fit_simultaneous(np.zeros((40, 40)), psf, dict(y=[20.0], x=[20.0], flux=[100.0]), 3, fixed=fixed)


def test_qfit_is_global_residual_based():
    # psf_photometry_simultaneous.jl:336-354
    psf = CircularGaussianPSF(fwhm=2.0)
    rng = np.random.default_rng(5)
    src = simulate_sources((64, 64), 3, rng=rng, flux=(500.0, 800.0), min_separation=6, border=8)
    img = np.zeros((64, 64))
    render_sources(img, psf, src["y"], src["x"], src["flux"], model_radius=5)
    r = orc_fit_simultaneous(img, psf, dict(y=src["y"], x=src["x"], flux=src["flux"]), 5,
                             fixed={"fwhm": 2.0, "bkg": 0.0}, max_iter=40, model_rad=5)
    for i in range(3):
        assert r.valid[i]
        ylo, yhi = max(int(np.floor(r.y[i] - 5)), 1), min(int(np.ceil(r.y[i] + 5)), 64)
        xlo, xhi = max(int(np.floor(r.x[i] - 5)), 1), min(int(np.ceil(r.x[i] + 5)), 64)
        want = np.abs(r.residual[ylo - 1:yhi, xlo - 1:xhi]).sum() / r.flux[i]
        assert r.qfit[i] == pytest.approx(want, rel=1e-10)


def crowded_gaussian(seed, shape=(200, 200), n=60):
    rng = np.random.default_rng(seed)
    psf = CircularGaussianPSF(fwhm=2.0)
    src = simulate_sources(shape, n, rng=rng, flux=(200.0, 3000.0), flux_distribution="powerlaw", flux_power=2.0,
                           min_separation=2, border=10)
    img = np.full(shape, 50.0)
    render_sources(img, psf, src["y"], src["x"], src["flux"], model_radius=6)
    add_noise(img, rng=rng, noise="poisson_gaussian", read_noise=2.0, gain=1.0)
    return img - 50.0, psf, src


def test_per_star_convergence_non_uniform_and_frozen_stable():
    # :407-424 and :426-453
    img, psf, src = crowded_gaussian(99)
    cat = dict(y=src["y"], x=src["x"], flux=src["flux"].copy())
    fixed = {"fwhm": 2.0, "bkg": 0.0}
    r1 = orc_fit_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=10, model_rad=5)
    r2 = orc_fit_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=25, model_rad=5)
    g = r2.valid
    assert g.sum() > 0.5 * g.size
    assert np.any(r2.n_iter[g] < r2.n_passes)
    assert len(np.unique(r2.n_iter[g])) > 1
    early = [i for i in range(g.size) if r1.valid[i] and r2.valid[i] and 0 < r2.n_iter[i] <= 10]
    assert len(early) > 0
    for i in early:
        assert r1.y[i] == pytest.approx(r2.y[i], abs=1e-8)
        assert r1.x[i] == pytest.approx(r2.x[i], abs=1e-8)
        assert r1.flux[i] == pytest.approx(r2.flux[i], rel=1e-8)


def test_model_radii_scalar_and_auto():
    # :466-483
    psf = CircularGaussianPSF(fwhm=2.5)
    w = np.full(4000, 1 / 125.0)
    fl = np.array([50, 500, 5000, 50000, 500000], dtype=float)
    rr = orc_model_radii_auto_gaussian(2.5, 1.0, 2, 20, w, fl)
    assert np.all(np.diff(rr) >= 0) and np.all((2 <= rr) & (rr <= 20))
    assert rr[0] == 2 and rr[-1] > rr[0]
    assert np.all(orc_model_radii_auto_gaussian(2.5, 3.0, 2, 20, w, fl) <= rr)
    # scalar path through the fit: clamp(ceil(model_rad), R_fit, R_cap)
    img = np.zeros((40, 40))
    cat = dict(y=[20.0], x=[20.0], flux=[100.0])
    fixed = {"fwhm": 2.5, "bkg": 0.0}
    for mr, want in [(7.0, 7), (1.0, 3), (3.2, 4)]:
        r = orc_fit_simultaneous(img + 1e-3, psf, cat, 3, fixed=fixed, model_rad=mr, max_iter=1, debug=True)
        assert r.debug["model_R"][0] == want


def test_fit_star_noiseless_recovery_gaussian():
    # psf_fitting_tests.jl:243-264
    truth = CircularGaussianPSF(y=15.3, x=16.8, fwhm=2.7, flux=1200.0, bkg=11.0)
    yy, xx = np.meshgrid(np.arange(1, 32), np.arange(1, 32), indexing="ij")
    img = truth.evaluate(yy.astype(float), xx.astype(float))
    init = CircularGaussianPSF(y=15.0, x=17.1, fwhm=2.4, flux=1000.0, bkg=10.0)
    best, res = orc_fit_star(init, img)
    assert res.converged
    for k in ("y", "x", "fwhm", "flux", "bkg"):
        assert getattr(best, k) == pytest.approx(getattr(truth, k), rel=1e-7, abs=1e-7)


def test_fit_star_gridded_four_corner_recovery():
    # psf_fit_parity_tests.jl:449-518 (inds not starting at 1, all four corners active)
    stampsize, c = 15, 8.0
    i = np.arange(1, 16)[:, None]
    j = np.arange(1, 16)[None, :]
    mk = lambda s2: ImagePSF(np.exp(-((i - c) ** 2 + (j - c) ** 2) / s2))
    nodes = [mk(5.0), mk(20.0), mk(20.0), mk(5.0)]
    gy, gx = [950.0, 950.0, 1010.0, 1010.0], [1200.0, 1275.0, 1200.0, 1275.0]
    truth = dict(y=1001.4, x=1240.7, flux=250.0, bkg=4.0)
    g = GriddedPSFModel(nodes, gy, gx, y=1000.9, x=1241.2, flux=230.0, bkg=4.4)
    img = np.zeros((1010, 1250))
    from oracle import orc_psf_eval
    yy, xx = np.meshgrid(np.arange(991, 1011), np.arange(1231, 1251), indexing="ij")
    f = orc_psf_eval(g, truth["y"], truth["x"], truth["flux"], truth["bkg"], yy.ravel().astype(float),
                     xx.ravel().astype(float), grad=False)
    img[990:1010, 1230:1250] = f.reshape(yy.shape)
    best, res = orc_fit_star(g, img, ((991, 1010), (1231, 1250)), inv_var=np.ones_like(img), x_tol=1e-7,
                             max_iter=100)
    assert res.converged
    for k in ("y", "x", "flux", "bkg"):
        assert getattr(best, k) == pytest.approx(truth[k], rel=1e-7, abs=1e-7)
    best2, res2 = orc_fit_star(g, img, ((991, 1010), (1231, 1250)), fixed={"bkg": 4.0}, x_tol=1e-7, max_iter=100)
    assert best2.bkg == 4.0
    assert best2.flux == pytest.approx(250.0, rel=1e-6)


def test_fit_star_inv_var_masking_and_errors():
    # psf_fitting_tests.jl:397-425 and _prepare_fit_star_inputs (psf_fitting.jl:61-90)
    truth = CircularGaussianPSF(y=8.2, x=7.6, fwhm=2.0, flux=500.0, bkg=3.0)
    yy, xx = np.meshgrid(np.arange(1, 16), np.arange(1, 16), indexing="ij")
    img = truth.evaluate(yy.astype(float), xx.astype(float))
    iv = np.ones_like(img)
    img[2, 3] = 1e6  # masked outlier
    iv[2, 3] = 0.0
    init = CircularGaussianPSF(y=8.0, x=8.0, fwhm=2.0, flux=400.0, bkg=3.0)
    best, res = orc_fit_star(init, img, inv_var=iv, fixed={"fwhm": 2.0})
    assert best.flux == pytest.approx(500.0, rel=1e-6)
    with pytest.raises(ArgumentError, match="too few valid"):
        orc_fit_star(init, img, inv_var=np.zeros_like(img))
