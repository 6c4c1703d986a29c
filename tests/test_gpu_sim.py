"""GPU simultaneous fit (through the C-ABI) vs the oracle on the same seeded inputs.

Parity bar: integer structures (active set / Morton order, stamp pixel
indices, model radii, union size) bit-exact; for stars valid and converged
in both, |dy|, |dx| <= 1e-4 px and |dflux|/flux <= 1e-5 (FP64 device path).
"""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF
from crowdphot_b200.simulate import (add_noise, crowded_field, moffat_epsf, render_sources, simulate_sources)
from oracle import orc_fit_simultaneous

pytestmark = pytest.mark.gpu

POS_TOL = 1e-4
FLUX_TOL = 1e-5


def parity_report(g, o):
    both = g.valid & o.valid & g.converged & o.converged
    same = both & (g.n_iter == o.n_iter)
    dy = np.abs(g.y - o.y)
    dx = np.abs(g.x - o.x)
    df = np.abs(g.flux / o.flux - 1)
    bad = same & ((dy > POS_TOL) | (dx > POS_TOL) | (df > FLUX_TOL))
    return both, same, dy, dx, df, bad


def assert_parity(g, o, min_same_frac=0.9):
    assert np.array_equal(g.valid, o.valid) or (g.valid != o.valid).sum() <= 0.01 * len(g.valid)
    both, same, dy, dx, df, bad = parity_report(g, o)
    assert both.sum() > 0
    assert same.sum() >= min_same_frac * both.sum(), f"freeze iterations differ for {both.sum() - same.sum()} stars"
    assert bad.sum() == 0, (f"{bad.sum()} stars outside the gates: max dy {dy[same].max():.3g} "
                            f"dx {dx[same].max():.3g} dflux {df[same].max():.3g}")


def c1_field(seed=1001, n=200, shape=(256, 256)):
    """256^2 Float64, 200 stars, CircularGaussianPSF FWHM 2.5, flat background 100 + Poisson."""
    rng = np.random.default_rng(seed)
    psf = CircularGaussianPSF(fwhm=2.5)
    src = simulate_sources(shape, n, rng=rng, flux=(1e2, 1e5), flux_distribution="loguniform")
    model = np.zeros(shape)
    render_sources(model, psf, src["y"], src["x"], src["flux"], model_radius=7)
    img = add_noise(model + 100.0, rng=rng, noise="poisson", gain=1.0)
    iv = 1.0 / (100.0 + model)
    init = dict(y=src["y"] + rng.normal(0, 0.3, n), x=src["x"] + rng.normal(0, 0.3, n),
                flux=src["flux"] * rng.uniform(0.9, 1.1, n))
    return img, np.full(shape, 100.0), iv, psf, src, init


def test_c1_config_parity():
    img, bkg, iv, psf, src, init = c1_field()
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=20,
              linear_tol=1e-8, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 7, **kw)
    o = orc_fit_simultaneous(img, psf, init, 7, **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert np.array_equal(g.debug["model_R"], o.debug["model_R"])
    assert g.stats["n_union"] == o.stats["n_union"]
    assert g.n_failed == o.n_failed
    assert_parity(g, o)


def test_crowded_epsf_parity_float32():
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1002, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 12, **kw)
    o = orc_fit_simultaneous(img, psf, init, 12, **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert g.stats["n_union"] == o.stats["n_union"]
    assert_parity(g, o, min_same_frac=0.8)


def test_edges_masks_and_nan_pixels_bit_exact_structures():
    rng = np.random.default_rng(3)
    psf = CircularGaussianPSF(fwhm=2.0)
    shape = (70, 90)
    n = 120
    ys = rng.uniform(-3, shape[0] + 3, n)
    xs = rng.uniform(-3, shape[1] + 3, n)
    ys[:4] = [0.5, 1.5, 2.5, 69.5]  # exact half-pixel anchors (round half to even)
    fs = rng.uniform(100, 2000, n)
    img = np.zeros(shape)
    render_sources(img, psf, ys, xs, fs, model_radius=5)
    img += rng.normal(0, 1, shape)
    iv = np.ones(shape)
    iv[10:20, 30:45] = 0.0
    iv[40, :] = np.nan
    img[5, 5] = np.nan
    ys[7] = np.nan
    good = (np.round(ys) >= 0) | np.isnan(ys)
    cat = dict(y=ys[good], x=np.abs(xs[good]), flux=fs[good])
    kw = dict(fixed={"fwhm": 2.0, "bkg": 0.0}, inv_var=iv, model_rad=6, max_iter=8, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, cat, 4, **kw)
    o = orc_fit_simultaneous(img, psf, cat, 4, **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert g.stats["n_union"] == o.stats["n_union"]
    assert g.n_failed == o.n_failed and g.n_failed > 0
    assert_parity(g, o, min_same_frac=0.8)


@pytest.mark.parametrize("kind", ["gaussian", "gridded"])
def test_isolated_noiseless_truth(kind):
    from test_oracle_fit import gaussian_node_psf, isolated_field
    psf = CircularGaussianPSF(fwhm=2.0) if kind == "gaussian" else gaussian_node_psf()
    fixed = {"fwhm": 2.0, "bkg": 0.0} if kind == "gaussian" else {"bkg": 0.0}
    img, src = isolated_field(psf)
    cat = dict(y=src["y"], x=src["x"], flux=np.full(5, 400.0))
    r = cpb.fit_all_stars_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=40, inner_iterations=10,
                                       x_tol=1e-8, model_rad=5)
    assert r.valid.all()
    np.testing.assert_allclose(r.flux, src["flux"], rtol=1e-10)
    np.testing.assert_allclose(r.y, src["y"], atol=1e-10)
    np.testing.assert_allclose(r.x, src["x"], atol=1e-10)
    o = orc_fit_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=40, inner_iterations=10, x_tol=1e-8,
                             model_rad=5)
    # noiseless: the reweighted covariance scales by cost/dof and that cost is pure rounding
    # (~1e-20), so the errors agree only to the relative size of that rounding
    np.testing.assert_allclose(r.flux_err, o.flux_err, rtol=1e-3)
    np.testing.assert_allclose(r.residual, o.residual, atol=1e-8)


def test_errors_chisq_qfit_match_oracle():
    img, bkg, iv, psf, src, init = c1_field(seed=77, n=60, shape=(128, 128))
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=20)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 7, **kw)
    o = orc_fit_simultaneous(img, psf, init, 7, **kw)
    both, same, *_ = parity_report(g, o)
    np.testing.assert_allclose(g.flux_err[same], o.flux_err[same], rtol=1e-4)
    np.testing.assert_allclose(g.y_err[same], o.y_err[same], rtol=1e-4)
    np.testing.assert_allclose(g.chisq[same], o.chisq[same], rtol=1e-3)
    np.testing.assert_allclose(g.qfit[same], o.qfit[same], rtol=1e-3)
    assert np.isfinite(g.spread_model[same]).all()
    np.testing.assert_allclose(g.spread_model[same], o.spread_model[same], rtol=0, atol=1e-4)
    np.testing.assert_allclose(g.spread_model_err[same], o.spread_model_err[same], rtol=1e-3)


def test_contract_errors_empty_and_failures_on_device():
    psf = CircularGaussianPSF(fwhm=2.0)
    img = np.zeros((64, 64))
    cat = dict(y=[32.0], x=[32.0], flux=[500.0])
    with pytest.raises(ArgumentError, match="fits only"):
        cpb.fit_all_stars_simultaneous(img, psf, cat, 5, model_rad=5)
    with pytest.raises(ArgumentError, match="LevenbergDamping"):
        cpb.fit_all_stars_simultaneous(img, psf, cat, 5, fixed={"fwhm": 2.0, "bkg": 0.0}, damping="levenberg",
                                       model_rad=5)
    r = cpb.fit_all_stars_simultaneous(np.zeros((16, 16)), psf, dict(y=[], x=[], flux=[]), 5,
                                       fixed={"fwhm": 2.0, "bkg": 0.0})
    assert r.flux.size == 0 and r.n_passes == 0
    bad = np.zeros((32, 32))
    bad[4, 4] = np.nan
    with pytest.raises(ArgumentError, match="non-finite"):
        cpb.fit_all_stars_simultaneous(bad, psf, dict(y=[16.0], x=[16.0], flux=[100.0]), 5,
                                       fixed={"fwhm": 2.0, "bkg": 0.0}, model_rad=5)
    iv = np.ones((32, 32))
    iv[9:22, 9:22] = 0
    r = cpb.fit_all_stars_simultaneous(np.zeros((32, 32)), psf, dict(y=[16.0], x=[16.0], flux=[100.0]), 5,
                                       fixed={"fwhm": 2.0, "bkg": 0.0}, inv_var=iv, model_rad=5)
    assert r.n_failed == 1 and not r.valid[0]


def test_deterministic_bitwise():
    img, bkg, iv, psf, src, init = c1_field(seed=5, n=80, shape=(128, 128))
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=10)
    a = cpb.fit_all_stars_simultaneous(img, psf, init, 7, **kw)
    b = cpb.fit_all_stars_simultaneous(img, psf, init, 7, **kw)
    assert np.array_equal(a.y, b.y) and np.array_equal(a.x, b.x) and np.array_equal(a.flux, b.flux)
    assert np.array_equal(a.residual, b.residual)


def test_mixed_precision_form_vs_fp64_oracle():
    """Mixed form (FP32 stamps / model values / products, FP64 solver state) against the
    FP64 oracle on the crowded ePSF field.  A truncated, freeze-as-you-go fit of a
    crowded field is sensitive to its trajectory: the oracle itself moves by
    ~1e-5 (median) when its initial guesses change by 1e-7 relative.  The mixed
    form must stay within that intrinsic spread (per output, median and p99)."""
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1002, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 12, precision="mixed", **kw)
    o = orc_fit_simultaneous(img, psf, init, 12, **kw)
    rng = np.random.default_rng(0)
    init2 = {k: v * (1 + 1e-7 * rng.standard_normal(v.size)) for k, v in init.items()}
    o2 = orc_fit_simultaneous(img, psf, init2, 12, **kw)
    both, same, dy, dx, df, bad = parity_report(g, o)
    _, same2, dy2, dx2, df2, _ = parity_report(o2, o)
    print(f"mixed vs FP64 oracle: {same.sum()}/{both.sum()} same freeze; dflux median/p99/max "
          f"{np.median(df[same]):.2e}/{np.percentile(df[same], 99):.2e}/{df[same].max():.2e}; dy "
          f"{np.median(dy[same]):.2e}/{np.percentile(dy[same], 99):.2e}; oracle spread under 1e-7 init "
          f"perturbation: dflux {np.median(df2[same2]):.2e}/{np.percentile(df2[same2], 99):.2e}, dy "
          f"{np.median(dy2[same2]):.2e}/{np.percentile(dy2[same2], 99):.2e}")
    assert same.sum() >= 0.8 * both.sum()
    for a_, b_ in ((df, df2), (dy, dy2), (dx, dx2)):
        assert np.median(a_[same]) <= 2 * np.median(b_[same2]) + 1e-7
        assert np.percentile(a_[same], 99) <= 2 * np.percentile(b_[same2], 99) + 1e-6


@pytest.mark.parametrize("kind", ["gaussian", "gridded"])
def test_mixed_precision_isolated_noiseless_truth(kind):
    from test_oracle_fit import gaussian_node_psf, isolated_field
    psf = CircularGaussianPSF(fwhm=2.0) if kind == "gaussian" else gaussian_node_psf()
    fixed = {"fwhm": 2.0, "bkg": 0.0} if kind == "gaussian" else {"bkg": 0.0}
    img, src = isolated_field(psf)
    cat = dict(y=src["y"], x=src["x"], flux=np.full(5, 400.0))
    r = cpb.fit_all_stars_simultaneous(img, psf, cat, 5, fixed=fixed, max_iter=40, x_tol=1e-8, model_rad=5,
                                       precision="mixed")
    assert r.valid.all()
    np.testing.assert_allclose(r.flux, src["flux"], rtol=2e-6)
    np.testing.assert_allclose(r.y, src["y"], atol=2e-5)
    np.testing.assert_allclose(r.x, src["x"], atol=2e-5)


@pytest.mark.parametrize("case", ["gaussian", "epsf"])
def test_model_rad_auto_radii_bit_exact_and_parity(case):
    """model_rad = :auto (the reference's default): per-star model radii from the
    unit PSF's curve of growth and the weight noise (_model_radii, :209-243) --
    bit-exact against the oracle -- and the fit's parity gates with those radii."""
    if case == "gaussian":
        img, bkg, iv, psf, src, init = c1_field(seed=21, n=150, shape=(160, 160))
        kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, max_iter=20, debug=True)
        R = 3
    else:
        psf = moffat_epsf()
        img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1012, psf=psf, dtype=np.float32)
        kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, debug=True)
        R = 8
    g = cpb.fit_all_stars_simultaneous(img, psf, init, R, model_rad="auto", **kw)
    o = orc_fit_simultaneous(img, psf, init, R, model_rad="auto", **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["model_R"], o.debug["model_R"])
    assert len(np.unique(o.debug["model_R"])) > 1  # radii really vary with flux
    assert_parity(g, o, min_same_frac=0.8)


def test_spread_model_parity_and_sequential_agreement():
    """spread_model on the device: the reference's simultaneous-vs-sequential test
    (test/photometry/psf_photometry_simultaneous.jl:356-383), the ePSF path (the disk
    width from the gridded PSF's effective area) against the oracle, a 30 px fit
    radius and the off switch."""
    from test_oracle_spread import FW, PSF
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
    rseq = cpb.fit_all_stars(sub, PSF, cat, 7, fixed=fixed, n_passes=3, max_iter=100, inv_var=iv)
    rsim = cpb.fit_all_stars_simultaneous(sub, PSF, cat, 7, fixed=fixed, max_iter=40, inv_var=iv)
    osim = orc_fit_simultaneous(sub, PSF, cat, 7, fixed=fixed, max_iter=40, inv_var=iv)
    np.testing.assert_allclose(rsim.spread_model, osim.spread_model, rtol=0, atol=1e-6)
    np.testing.assert_allclose(rsim.spread_model_err, osim.spread_model_err, rtol=1e-5)
    for i in range(3):
        assert abs(rseq.spread_model[i]) < 3e-3 and abs(rsim.spread_model[i]) < 3e-3
        assert abs(rseq.spread_model[i] - rsim.spread_model[i]) < 2e-3
    assert rseq.spread_model[3] > 5e-3 and rsim.spread_model[3] > 5e-3
    off = cpb.fit_all_stars_simultaneous(sub, PSF, cat, 7, fixed=fixed, max_iter=40, inv_var=iv, spread_model_fwhm=0)
    assert np.isnan(off.spread_model).all() and np.isfinite(off.qfit).all()
    # ePSF, float32, crowded; and a 30 px fit radius
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(128, 128, 200, seed=1009, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, max_iter=10)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 12, **kw)
    o = orc_fit_simultaneous(img, psf, init, 12, **kw)
    both, same, *_ = parity_report(g, o)
    assert np.isfinite(g.spread_model[same]).all()
    np.testing.assert_allclose(g.spread_model[same], o.spread_model[same], rtol=0, atol=1e-4)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=30, max_iter=3)
    sel = {k: np.asarray(v)[:12] for k, v in init.items()}
    g = cpb.fit_all_stars_simultaneous(img, psf, sel, 30, **kw)
    o = orc_fit_simultaneous(img, psf, sel, 30, **kw)
    both, same, *_ = parity_report(g, o)
    assert same.sum() > 0
    np.testing.assert_allclose(g.spread_model[same], o.spread_model[same], rtol=0, atol=1e-4)


def four_node_epsf():
    """A 2 x 2 grid of Moffat ePSF nodes (FWHM 2.4 .. 3.2 px) over a 128^2 field: the
    general (several-node) stamp path."""
    nodes = [moffat_epsf(fwhm=f, size=121).psfs[0] for f in (2.4, 2.8, 2.8, 3.2)]
    return cpb.GriddedPSFModel(nodes, [20.0, 20.0, 110.0, 110.0], [20.0, 110.0, 20.0, 110.0])


def test_four_node_gridded_parity_and_large_radii():
    """Multi-node GriddedPSFModel against the oracle: the block-per-star stamp kernels,
    spread_model from the blended PSF's effective area; then a 26 px fit radius and a
    50 px model radius (the 512-thread stamp kernel and the value-only render)."""
    from oracle import orc_psf_eval
    psf = four_node_epsf()
    rng = np.random.default_rng(1013)
    n, shape = 150, (128, 128)
    src = simulate_sources(shape, n, rng=rng, flux=(3e2, 3e4), flux_distribution="loguniform")
    model = np.zeros(shape)
    for y, x, f in zip(src["y"], src["x"], src["flux"]):
        ya, yb = max(int(y) - 15, 1), min(int(y) + 15, shape[0])
        xa, xb = max(int(x) - 15, 1), min(int(x) + 15, shape[1])
        yy, xx = np.meshgrid(np.arange(ya, yb + 1), np.arange(xa, xb + 1), indexing="ij")
        v = orc_psf_eval(psf, y, x, f, 0.0, yy.ravel().astype(float), xx.ravel().astype(float), grad=False)
        model[ya - 1:yb, xa - 1:xb] += v.reshape(yy.shape)
    bkg = np.full(shape, 50.0)
    img = add_noise(model + bkg, rng=rng, noise="poisson", gain=1.0)
    iv = 1.0 / (bkg + model)
    init = dict(y=src["y"] + rng.normal(0, 0.3, n), x=src["x"] + rng.normal(0, 0.3, n),
                flux=src["flux"] * rng.uniform(0.9, 1.1, n))
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, max_iter=12, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 8, **kw)
    o = orc_fit_simultaneous(img, psf, init, 8, **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert_parity(g, o, min_same_frac=0.8)
    both, same, *_ = parity_report(g, o)
    np.testing.assert_allclose(g.spread_model[same], o.spread_model[same], rtol=0, atol=1e-4)
    sel = {k: np.asarray(v)[:10] for k, v in init.items()}
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=50, max_iter=10, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, sel, 26, **kw)
    o = orc_fit_simultaneous(img, psf, sel, 26, **kw)
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert np.array_equal(g.debug["model_R"], o.debug["model_R"])
    assert_parity(g, o, min_same_frac=0.5)
