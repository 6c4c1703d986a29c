"""GPU simultaneous fit (through the C-ABI) vs the oracle on the same seeded inputs.

Parity bar: integer structures (active set / Morton order, stamp pixel
indices, model radii, union size) bit-exact; for stars valid and converged
in both, |dy|, |dx| <= 1e-4 px and |dflux|/flux <= 1e-5 (FP64 device path).
"""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF
from crowdphot_b200.simulate import (add_noise, c1_field, crowded_field, moffat_epsf, render_sources,
                                      simulate_sources)
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


def assert_parity(g, o, min_same_frac=1.0, max_valid_diff=0, tag=""):
    """Gates for stars valid and converged in both fits that freeze on the same
    iteration; `min_same_frac` (just under the measured fraction of each test) bounds
    how many may freeze on different iterations, and their deviations are printed."""
    nvd = int((g.valid != o.valid).sum())
    assert nvd <= max_valid_diff, f"valid flags differ for {nvd} stars"
    both, same, dy, dx, df, bad = parity_report(g, o)
    assert both.sum() > 0
    diff = both & ~same
    msg = (f"parity {tag}: {int(same.sum())}/{int(both.sum())} same freeze iteration "
           f"({same.sum() / both.sum():.4f}); same: max dy {dy[same].max():.2e} dx {dx[same].max():.2e} "
           f"dflux {df[same].max():.2e}")
    if diff.any():
        msg += (f"; different freeze ({int(diff.sum())}): max dy {dy[diff].max():.2e} dx {dx[diff].max():.2e} "
                f"dflux {df[diff].max():.2e}")
    print(msg)
    assert same.sum() >= min_same_frac * both.sum(), msg
    assert bad.sum() == 0, (f"{bad.sum()} stars outside the gates: max dy {dy[same].max():.3g} "
                            f"dx {dx[same].max():.3g} dflux {df[same].max():.3g}")


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
    assert_parity(g, o, tag="c1")


def test_crowded_epsf_parity_float32():
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1002, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 12, **kw)
    o = orc_fit_simultaneous(img, psf, init, 12, **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert g.stats["n_union"] == o.stats["n_union"]
    assert_parity(g, o, tag="crowded_f32")


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
    assert_parity(g, o, tag="edges")


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


def _perturbed(img, seed):
    """The image times (1 + 1e-7 N(0, 1)), rounded to its own element type: a change
    at the input's own rounding (about one ulp of a Float32 image on half the pixels)."""
    g = np.random.default_rng(seed)
    return (img.astype(np.float64) * (1 + 1e-7 * g.standard_normal(img.shape))).astype(img.dtype)


def test_mixed_precision_form_follows_the_fp64_trajectory():
    """Mixed form (FP32 stamps, model values and LSQR pixel vectors; FP64 sums,
    solver state, 3x3 solves and chi^2) against the FP64 oracle on the crowded ePSF
    field, twelve Gauss-Newton iterations with freezing and the global stops off, so
    that both take the same steps.  Stars whose result the data do not fix move when
    the input moves by its own rounding; the stars the oracle reproduces to a tenth of
    the gates under two such perturbations form the stable set, and there the mixed
    form meets the gates themselves (1e-4 px, 1e-5 relative flux).  (The default
    tolerances stop a crowded fit on global tests -- f_tol, the gradient cosine --
    whose outcome can flip under FP32 rounding and move every star by a step; the
    bench reports that comparison at full size.)"""
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1002, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, max_iter=12, x_tol=0.0, f_tol=0.0,
              g_tol=0.0)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 12, precision="mixed", **kw)
    o = orc_fit_simultaneous(img, psf, init, 12, **kw)
    assert g.n_passes == o.n_passes == 12
    fitted = o.valid & g.valid
    stable = fitted.copy()
    for seed in (11, 12):
        op = orc_fit_simultaneous(_perturbed(img, seed), psf, init, 12, **kw)
        stable &= op.valid
        stable &= np.abs(op.flux / o.flux - 1) <= 0.1 * FLUX_TOL
        stable &= np.maximum(np.abs(op.y - o.y), np.abs(op.x - o.x)) <= 0.1 * POS_TOL
    df = np.abs(g.flux / o.flux - 1)
    dp = np.maximum(np.abs(g.y - o.y), np.abs(g.x - o.x))
    print(f"mixed vs FP64 oracle, 12 iterations: stable set {int(stable.sum())} of {int(fitted.sum())} valid; on "
          f"it dflux median/p99/max {np.median(df[stable]):.2e}/{np.percentile(df[stable], 99):.2e}/"
          f"{df[stable].max():.2e}, dpos max {dp[stable].max():.2e}; all valid: dflux within 1e-5 "
          f"{np.mean(df[fitted] <= FLUX_TOL):.3f}")
    assert stable.sum() >= 0.3 * fitted.sum()
    assert df[stable].max() <= FLUX_TOL and dp[stable].max() <= POS_TOL


def test_tight_tolerance_every_valid_star():
    """The reference's converged-mode comparison (test/photometry/psf_photometry_simultaneous.jl:270-274):
    with f_tol off and a tight x_tol both fits run to the same minimum, so every
    valid star -- not only those frozen on the same iteration -- meets the gates."""
    img, bkg, iv, psf, src, init = c1_field()
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=60,
              linear_tol=1e-8, x_tol=1e-10, f_tol=0.0)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 7, **kw)
    o = orc_fit_simultaneous(img, psf, init, 7, **kw)
    assert np.array_equal(g.valid, o.valid)
    v = g.valid
    dy, dx, df = np.abs(g.y - o.y)[v], np.abs(g.x - o.x)[v], np.abs(g.flux / o.flux - 1)[v]
    print(f"tight: {int(v.sum())} valid, {int((g.converged & v).sum())} converged; max dy {dy.max():.2e} "
          f"dx {dx.max():.2e} dflux {df.max():.2e}")
    assert dy.max() <= POS_TOL and dx.max() <= POS_TOL and df.max() <= FLUX_TOL


def test_mixed_precision_refinement_reaches_the_fp64_minimum():
    """refine_iters: FP64 Gauss-Newton iterations after the FP32-stamp loop.  Run to a
    minimum of the whole field (freezing and the global stops off, 120 iterations,
    where the FP64 fit no longer moves), the FP32-stamp loop stalls where its accept
    test no longer resolves the cost (median flux deviation from the oracle ~3e-8);
    twenty FP64 refinement iterations bring the median to FP64 rounding and every
    valid star whose nearest neighbour is at least 3 px away (pairs closer than about
    a FWHM converge slowly at any precision) inside the gates."""
    img, bkg, iv, psf, src, init = c1_field()
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=120,
              linear_tol=1e-10, x_tol=0.0, f_tol=0.0, g_tol=0.0)
    g = cpb.fit_all_stars_simultaneous(img, psf, init, 7, precision="mixed", refine_iters=20, **kw)
    m = cpb.fit_all_stars_simultaneous(img, psf, init, 7, precision="mixed", **kw)
    o = orc_fit_simultaneous(img, psf, init, 7, **kw)
    assert np.array_equal(g.valid, o.valid) and np.array_equal(m.valid, o.valid)
    d = np.hypot(src["y"][:, None] - src["y"][None], src["x"][:, None] - src["x"][None]) + 1e9 * np.eye(len(src["y"]))
    apart = g.valid & (d.min(1) >= 3.0)
    df = lambda r: np.abs(r.flux / o.flux - 1)
    dp = lambda r: np.maximum(np.abs(r.y - o.y), np.abs(r.x - o.x))
    print(f"minimum: mixed median dflux {np.median(df(m)[g.valid]):.1e}, refined {np.median(df(g)[g.valid]):.1e}; "
          f"{int(apart.sum())} stars >= 3 px apart: refined max dflux {df(g)[apart].max():.1e} dpos "
          f"{dp(g)[apart].max():.1e}; passes {g.n_passes} (mixed {m.n_passes}, oracle {o.n_passes})")
    assert np.median(df(g)[g.valid]) <= 1e-12 < np.median(df(m)[g.valid])
    assert df(g)[apart].max() <= FLUX_TOL and dp(g)[apart].max() <= POS_TOL
    assert g.n_passes == m.n_passes + 20 == o.n_passes + 20
    with pytest.raises(ArgumentError, match="refine_iters"):
        cpb.fit_all_stars_simultaneous(img, psf, init, 7, precision="mixed", refine_iters=-1, **kw)


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
    assert_parity(g, o, tag=f"auto_{case}")


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
    assert_parity(g, o, tag="four_node")
    both, same, *_ = parity_report(g, o)
    np.testing.assert_allclose(g.spread_model[same], o.spread_model[same], rtol=0, atol=1e-4)
    sel = {k: np.asarray(v)[:10] for k, v in init.items()}
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=50, max_iter=10, debug=True)
    g = cpb.fit_all_stars_simultaneous(img, psf, sel, 26, **kw)
    o = orc_fit_simultaneous(img, psf, sel, 26, **kw)
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert np.array_equal(g.debug["model_R"], o.debug["model_R"])
    assert_parity(g, o, tag="large_radii")


@pytest.mark.parametrize("case", ["c1", "crowded_epsf"])
def test_lsmr_solver_parity(case):
    """solver = :lsmr (krylov_solve! with the LSMR workspace, :1222-1224): the same
    Golub-Kahan kernels as LSQR with LSMR's rotations and h / hbar / x updates,
    against the oracle's LSMR restatement -- integer structures bit-exact, the same
    parity gates as LSQR, and a result that differs from the LSQR fit (the solver
    really changed)."""
    if case == "c1":
        img, bkg, iv, psf, src, init = c1_field()
        kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=20,
                  linear_tol=1e-8, debug=True)
        R = 7
    else:
        psf = moffat_epsf()
        img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1002, psf=psf, dtype=np.float32)
        kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad=12, debug=True)
        R = 12
    g = cpb.fit_all_stars_simultaneous(img, psf, init, R, solver="lsmr", **kw)
    o = orc_fit_simultaneous(img, psf, init, R, solver="lsmr", **kw)
    assert np.array_equal(g.debug["active"], o.debug["active"])
    assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
    assert_parity(g, o, tag=f"lsmr_{case}")
    q = cpb.fit_all_stars_simultaneous(img, psf, init, R, **kw)
    assert np.max(np.abs(q.flux / g.flux - 1)[g.valid & q.valid]) > 0


@pytest.mark.parametrize("variant", [{"solver": "lsmr"}, {"model_rad": "auto"}, {"precision": "mixed"}],
                         ids=["lsmr", "auto_radii", "mixed"])
def test_routed_group_variants_equal_single_fits(variant):
    """The block-per-group kernel computes in FP64 with LSQR and one scalar model
    radius; solver = :lsmr, model_rad = :auto and the mixed form fit every group of
    a batch through the full-field path instead: each group equals its own single
    fit."""
    from crowdphot_b200.simulate import lm_groups
    psf = moffat_epsf()
    d = lm_groups(6, seed=77, psf=psf, kmax=5)
    offs, so = d["offsets"], d["star_offsets"]
    images, cats, ivs = [], [], []
    for gi in range(6):
        ny, nx = int(d["ny"][gi]), int(d["nx"][gi])
        a, b = int(so[gi]), int(so[gi + 1])
        images.append(d["pix"][offs[gi]:offs[gi] + ny * nx].reshape((ny, nx), order="F"))
        ivs.append(d["inv_var"][offs[gi]:offs[gi] + ny * nx].reshape((ny, nx), order="F"))
        cats.append(dict(y=d["y"][a:b], x=d["x"][a:b], flux=d["flux"][a:b]))
    kw = dict({"fixed": {"bkg": 0.0}, "model_rad": 12}, **variant)
    res = cpb.fit_all_stars_simultaneous_batch(images, psf, cats, 5, inv_vars=ivs, **kw)
    for gi in range(6):
        s = cpb.fit_all_stars_simultaneous(images[gi], psf, cats[gi], 5, inv_var=ivs[gi], **kw)
        assert np.array_equal(s.valid, res[gi].valid)
        ok = s.valid
        np.testing.assert_allclose(res[gi].flux[ok], s.flux[ok], rtol=1e-12)
        np.testing.assert_allclose(res[gi].y[ok], s.y[ok], rtol=0, atol=1e-12)
