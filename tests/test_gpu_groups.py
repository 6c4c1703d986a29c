"""Batched simultaneous fits of small star groups (cpb_fit_simultaneous_batch,
one thread block per group) against the oracle's fit_all_stars_simultaneous
run on each group alone, on the same seeded inputs.

Parity bar (FP64 device arithmetic), per group: active-star count, union size
and failure count bit-exact; for stars valid and converged in both with the
same freeze iteration, |dy|, |dx| <= 1e-4 px and |dflux|/flux <= 1e-5; errors
within 1e-4 relative; chi^2 and qfit within 1e-3 relative; spread_model within
1e-5 absolute and its error within 1e-3 relative (the disk width comes from
each group's first star's fitted position, so it moves with the fit).
"""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF
from crowdphot_b200.simulate import lm_groups, moffat_epsf, render_sources
from oracle import orc_fit_simultaneous

pytestmark = pytest.mark.gpu

POS_TOL = 1e-4
FLUX_TOL = 1e-5
C4_KW = dict(fixed={"bkg": 0.0}, model_rad=12)


def group_image(d, g, key="pix"):
    off, ny, nx = int(d["offsets"][g]), int(d["ny"][g]), int(d["nx"][g])
    return d[key][off:off + ny * nx].reshape((ny, nx), order="F")


def group_cat(d, g):
    s0, s1 = int(d["star_offsets"][g]), int(d["star_offsets"][g + 1])
    return dict(y=d["y"][s0:s1], x=d["x"][s0:s1], flux=d["flux"][s0:s1])


def run_batch(psf, d, fit_rad, **kw):
    return cpb.fit_groups_packed(psf, d["pix"], d["offsets"], d["ny"], d["nx"], d["star_offsets"], d["y"], d["x"],
                                 d["flux"], fit_rad, inv_var=d.get("inv_var"), background=d.get("bkg"), **kw)


def compare(d, out, psf, fit_rad, min_same=0.9, check_errors=True, **kw):
    G = len(d["ny"])
    same_all = both_all = 0
    worst = [0.0, 0.0, 0.0]
    for g in range(G):
        o = orc_fit_simultaneous(group_image(d, g), psf, group_cat(d, g), fit_rad,
                                 inv_var=None if d.get("inv_var") is None else group_image(d, g, "inv_var"),
                                 background=None if d.get("bkg") is None else group_image(d, g, "bkg"), **kw)
        s0, s1 = int(d["star_offsets"][g]), int(d["star_offsets"][g + 1])
        sl = slice(s0, s1)
        assert out["status"][g] == 0
        assert out["n_active"][g] == o.stats["n_active"], g
        assert out["n_union"][g] == o.stats["n_union"], g
        assert out["n_failed"][g] == o.n_failed, g
        gv, gc = out["valid"][sl].astype(bool), out["converged"][sl].astype(bool)
        assert (gv != o.valid).sum() <= max(1, 0.05 * (s1 - s0)), g
        both = gv & o.valid & gc & o.converged
        same = both & (out["n_iter"][sl] == o.n_iter)
        both_all += both.sum()
        same_all += same.sum()
        dy = np.abs(out["y"][sl] - o.y)[same]
        dx = np.abs(out["x"][sl] - o.x)[same]
        df = np.abs(out["flux"][sl] / o.flux - 1)[same]
        if same.any():
            worst = [max(worst[0], dy.max()), max(worst[1], dx.max()), max(worst[2], df.max())]
            assert dy.max() <= POS_TOL and dx.max() <= POS_TOL and df.max() <= FLUX_TOL, (g, dy.max(), df.max())
            np.testing.assert_allclose(out["spread_model"][sl][same], o.spread_model[same], rtol=0, atol=1e-5)
            np.testing.assert_allclose(out["spread_model_err"][sl][same], o.spread_model_err[same], rtol=1e-3,
                                       equal_nan=True)
            if check_errors:
                np.testing.assert_allclose(out["flux_err"][sl][same], o.flux_err[same], rtol=1e-4)
                np.testing.assert_allclose(out["y_err"][sl][same], o.y_err[same], rtol=1e-4)
                np.testing.assert_allclose(out["chisq"][sl][same], o.chisq[same], rtol=1e-3)
                np.testing.assert_allclose(out["qfit"][sl][same], o.qfit[same], rtol=1e-3)
        # stars the oracle left out of the solve keep the catalogue values on the device too
        untouched = ~o.valid & (o.flux == d["flux"][sl]) & (o.n_iter == 0)
        np.testing.assert_array_equal(out["flux"][sl][untouched], o.flux[untouched])
        np.testing.assert_array_equal(gv[untouched], False)
        assert np.isnan(out["spread_model"][sl][~gv]).all()
    assert both_all > 0
    assert same_all >= min_same * both_all, f"freeze iterations differ for {both_all - same_all} stars"
    print(f"groups: {same_all}/{both_all} stars compared; max dy {worst[0]:.2e} dx {worst[1]:.2e} "
          f"dflux {worst[2]:.2e}")


def test_c4_groups_match_oracle():
    psf = moffat_epsf()
    d = lm_groups(160, seed=1104)
    out = run_batch(psf, d, 5, residual=True, **C4_KW)
    assert out["n_kernel_groups"] == 160 and out["n_routed_groups"] == 0
    compare(d, out, psf, 5, **C4_KW)


def test_groups_residual_matches_oracle():
    psf = moffat_epsf()
    d = lm_groups(24, seed=7, kmax=6)
    out = run_batch(psf, d, 5, residual=True, **C4_KW)
    for g in range(24):
        o = orc_fit_simultaneous(group_image(d, g), psf, group_cat(d, g), 5, inv_var=group_image(d, g, "inv_var"),
                                 **C4_KW)
        s0, s1 = int(d["star_offsets"][g]), int(d["star_offsets"][g + 1])
        dpar = max(np.abs(out["y"][s0:s1] - o.y).max(), np.abs(out["x"][s0:s1] - o.x).max(),
                   np.abs(out["flux"][s0:s1] / o.flux - 1).max())
        if dpar > 1e-9:
            continue  # residual is compared where the fitted parameters agree to rounding
        r = out["residual"][d["offsets"][g]:d["offsets"][g] + d["ny"][g] * d["nx"][g]]
        np.testing.assert_allclose(r, o.residual.ravel(order="F"), atol=1e-6 * (1 + np.abs(o.residual).max()))


def test_groups_gaussian_float64_with_background():
    rng = np.random.default_rng(11)
    psf = CircularGaussianPSF(fwhm=2.5)
    G = 40
    k = rng.integers(2, 9, G)
    side = 8 * k + 17
    pix, iv, bk, ys, xs, fs, truth = [], [], [], [], [], [], []
    for g in range(G):
        sh = (int(side[g]), int(side[g]))
        y = rng.uniform(2, sh[0] - 1, k[g])
        x = rng.uniform(2, sh[1] - 1, k[g])
        f = np.exp(rng.uniform(np.log(300), np.log(3e4), k[g]))
        m = np.zeros(sh)
        render_sources(m, psf, y, x, f, model_radius=7)
        b = np.full(sh, 100.0)
        img = rng.poisson(m + b).astype(np.float64)
        pix.append(img.ravel(order="F"))
        iv.append((1.0 / (m + b)).ravel(order="F"))
        bk.append(b.ravel(order="F"))
        ys.append(y + rng.normal(0, 0.3, k[g]))
        xs.append(x + rng.normal(0, 0.3, k[g]))
        fs.append(f * rng.uniform(0.9, 1.1, k[g]))
    sizes = side.astype(np.int64) ** 2
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    d = dict(pix=np.concatenate(pix), inv_var=np.concatenate(iv), bkg=np.concatenate(bk), offsets=off,
             ny=side.astype(np.int32), nx=side.astype(np.int32), star_offsets=np.concatenate([[0], np.cumsum(k)]),
             y=np.concatenate(ys), x=np.concatenate(xs), flux=np.concatenate(fs))
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, model_rad=7, max_iter=20, linear_tol=1e-8)
    out = run_batch(psf, d, 7, **kw)
    compare(d, out, psf, 7, **kw)


def test_groups_edges_masks_empty_and_routed():
    """Empty groups, groups whose stars all miss the image, masked / NaN pixels, stars
    hanging over the edge, and one group of 70 stars (too many for one block: it goes
    through the full-field path) in the same batch."""
    rng = np.random.default_rng(5)
    psf = CircularGaussianPSF(fwhm=2.0)
    specs = [(40, 40, 0), (40, 40, 3), (50, 60, 6), (45, 45, 5), (120, 120, 70), (33, 33, 4)]
    pix, iv, ys, xs, fs = [], [], [], [], []
    for gi, (ny, nx, n) in enumerate(specs):
        if gi == 1:
            y = rng.uniform(-40, -20, n)
            x = rng.uniform(1, nx, n)
        elif gi == 3:
            y = np.array([1.2, 44.7, 20.0, 0.6, 23.0])
            x = np.array([1.4, 44.9, 0.8, 20.0, 46.6])
        else:
            y = rng.uniform(1, ny, n)
            x = rng.uniform(1, nx, n)
        f = rng.uniform(300, 5000, n)
        m = np.zeros((ny, nx))
        render_sources(m, psf, y, x, f, model_radius=6)
        img = m + rng.normal(0, 1.0, (ny, nx))
        w = np.ones((ny, nx))
        if gi == 2:
            w[10:18, 20:30] = 0.0
            w[30, :] = np.nan
            img[5, 5] = np.nan
        pix.append(img.ravel(order="F"))
        iv.append(w.ravel(order="F"))
        ys.append(y + rng.normal(0, 0.2, n))
        xs.append(x + rng.normal(0, 0.2, n))
        fs.append(f * rng.uniform(0.9, 1.1, n))
    ny_ = np.array([s[0] for s in specs], np.int32)
    nx_ = np.array([s[1] for s in specs], np.int32)
    sizes = ny_.astype(np.int64) * nx_
    d = dict(pix=np.concatenate(pix), inv_var=np.concatenate(iv), offsets=np.concatenate([[0], np.cumsum(sizes)[:-1]]),
             ny=ny_, nx=nx_, star_offsets=np.concatenate([[0], np.cumsum([s[2] for s in specs])]),
             y=np.concatenate(ys), x=np.concatenate(xs), flux=np.concatenate(fs))
    kw = dict(fixed={"fwhm": 2.0, "bkg": 0.0}, model_rad=6, max_iter=15)
    out = run_batch(psf, d, 4, residual=True, **kw)
    assert out["n_routed_groups"] == 1 and out["n_kernel_groups"] == len(specs) - 1
    assert out["n_passes"][0] == 0 and out["n_failed"][0] == 0
    assert out["n_active"][1] == 0 and out["n_failed"][1] == 3 and not out["valid"][0:3].any()
    compare(d, out, psf, 4, min_same=0.8, check_errors=False, **kw)


def test_group_argument_errors_are_per_group():
    psf = CircularGaussianPSF(fwhm=2.0)
    ny = nx = 30
    good = np.zeros((ny, nx))
    render_sources(good, psf, [15.2], [14.7], [800.0], model_radius=6)
    bad = good.copy()
    bad[3, 3] = np.nan
    d = dict(pix=np.concatenate([good.ravel(order="F"), bad.ravel(order="F"), good.ravel(order="F")]),
             offsets=np.array([0, ny * nx, 2 * ny * nx]), ny=np.full(3, ny, np.int32), nx=np.full(3, nx, np.int32),
             star_offsets=np.array([0, 1, 2, 4]), y=np.array([15.0, 15.0, 15.0, -0.6]),
             x=np.array([15.0, 15.0, 15.0, 10.0]), flux=np.array([700.0, 700.0, 700.0, 50.0]))
    kw = dict(fixed={"fwhm": 2.0, "bkg": 0.0}, model_rad=6)
    out = run_batch(psf, d, 5, **kw)
    assert list(out["status"]) == [0, -1, -1]
    assert list(out["error_kind"]) == [0, 1, 2]
    o = orc_fit_simultaneous(good, psf, dict(y=[15.0], x=[15.0], flux=[700.0]), 5, **kw)
    assert abs(out["flux"][0] / o.flux[0] - 1) < FLUX_TOL
    with pytest.raises(ArgumentError, match="non-finite"):
        cpb.fit_all_stars_simultaneous_batch([good, bad], psf, [dict(y=[15.0], x=[15.0], flux=[700.0])] * 2, 5, **kw)
    # the mixed form routes every group to the full-field fit: the same per-group
    # statuses, and group 0 equals its own single mixed fit
    outm = run_batch(psf, d, 5, precision="mixed", **kw)
    assert list(outm["status"]) == [0, -1, -1]
    sm = cpb.fit_all_stars_simultaneous(good, psf, dict(y=[15.0], x=[15.0], flux=[700.0]), 5, precision="mixed",
                                        **kw)
    np.testing.assert_allclose(outm["flux"][0], sm.flux[0], rtol=1e-12)


def test_groups_deterministic_and_equal_to_single_fits():
    psf = moffat_epsf()
    d = lm_groups(48, seed=99)
    a = run_batch(psf, d, 5, **C4_KW)
    b = run_batch(psf, d, 5, **C4_KW)
    for k in ("y", "x", "flux", "flux_err", "n_iter", "chisq", "spread_model", "spread_model_err"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    images = [group_image(d, g) for g in range(48)]
    ivs = [group_image(d, g, "inv_var") for g in range(48)]
    cats = [group_cat(d, g) for g in range(48)]
    res = cpb.fit_all_stars_simultaneous_batch(images, psf, cats, 5, inv_vars=ivs, **C4_KW)
    for g in (0, 17, 47):
        s = cpb.fit_all_stars_simultaneous(images[g], psf, cats[g], 5, inv_var=ivs[g], **C4_KW)
        ok = s.valid & s.converged & res[g].valid & res[g].converged & (s.n_iter == res[g].n_iter)
        assert ok.any()
        assert np.abs(s.y - res[g].y)[ok].max() <= POS_TOL
        assert np.abs(s.flux / res[g].flux - 1)[ok].max() <= FLUX_TOL
        assert np.abs(s.spread_model - res[g].spread_model)[ok].max() <= 1e-5
        assert res[g].n_passes == s.n_passes or ok.sum() >= 0.8 * len(ok)


def test_groups_spread_model_width_and_off_switch():
    """An explicit disk width replaces the per-group one (the same disk for every
    group); a non-positive or non-finite width, or no spread_model outputs,
    turns spread_model off without touching the fit."""
    psf = moffat_epsf()
    d = lm_groups(40, seed=321)
    for width in (3.0, 6.5):
        out = run_batch(psf, d, 5, spread_model_fwhm=width, **C4_KW)
        compare(d, out, psf, 5, check_errors=False, spread_model_fwhm=width, **C4_KW)
    base = run_batch(psf, d, 5, **C4_KW)
    for off in (0.0, -2.0, float("inf")):
        out = run_batch(psf, d, 5, spread_model_fwhm=off, **C4_KW)
        assert np.isnan(out["spread_model"]).all() and np.isnan(out["spread_model_err"]).all()
        for k in ("y", "x", "flux", "chisq", "qfit"):
            assert np.array_equal(out[k], base[k], equal_nan=True), k


def test_groups_disk_width_from_each_groups_first_star():
    """Each group's disk is sized from its own first star's fitted position
    (psf_photometry_simultaneous.jl:1363-1364): the batch equals, per group, a run
    given that width explicitly (computed on the host by the oracle's
    _spread_fwhm); the single-field path does the same."""
    from oracle import orc_spread_fwhm
    psf = moffat_epsf()
    d = lm_groups(12, seed=4242)
    out = run_batch(psf, d, 5, **C4_KW)
    for g in range(12):
        s0, s1 = int(d["star_offsets"][g]), int(d["star_offsets"][g + 1])
        if not out["valid"][s0:s1].any():
            continue
        f = orc_spread_fwhm(psf, out["y"][s0], out["x"][s0])
        sub = dict(pix=group_image(d, g).ravel(order="F"), inv_var=group_image(d, g, "inv_var").ravel(order="F"),
                   offsets=np.array([0]), ny=d["ny"][g:g + 1], nx=d["nx"][g:g + 1],
                   star_offsets=np.array([0, s1 - s0]), y=d["y"][s0:s1], x=d["x"][s0:s1], flux=d["flux"][s0:s1])
        ex = run_batch(psf, sub, 5, spread_model_fwhm=f, **C4_KW)
        np.testing.assert_allclose(ex["spread_model"], out["spread_model"][s0:s1], rtol=0, atol=1e-12,
                                   equal_nan=True)
        single = cpb.fit_all_stars_simultaneous(group_image(d, g), psf, group_cat(d, g), 5,
                                                inv_var=group_image(d, g, "inv_var"), **C4_KW)
        f1 = orc_spread_fwhm(psf, single.y[0], single.x[0])
        single_ex = cpb.fit_all_stars_simultaneous(group_image(d, g), psf, group_cat(d, g), 5,
                                                   inv_var=group_image(d, g, "inv_var"), spread_model_fwhm=f1,
                                                   **C4_KW)
        np.testing.assert_allclose(single_ex.spread_model, single.spread_model, rtol=0, atol=1e-12, equal_nan=True)
