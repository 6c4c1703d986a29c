"""The simultaneous fit through the checked build of the library
(lib/libcrowdphot_b200_checked.so: cpb_sim.cu compiled with -DCPB_CHECKED), in
which every stamp-rectangle load and store, and every shared-memory region slot
the J.v gather writes, is tested against its buffer's length; a failed test
skips the access and the call fails with the site's code.  Cases: image edges,
masked and NaN pixels, both precisions, model_rad = :auto, boxes meeting more
than 2 x 2 regions (the per-pair rectangle path), a 26 px fit box with a 50 px
model box.  The results must also equal the production build's within the
parity gates: the checks change no arithmetic."""
import os

import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import CircularGaussianPSF, _abi
from crowdphot_b200.simulate import c1_field, crowded_field, moffat_epsf, render_sources

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def checked():
    if not os.path.exists(_abi.CHECKED_LIB_PATH):
        pytest.fail("the checked library is not built (make -C crowdphot.jl_b200/csrc all)")
    ctx = cpb.Context(0, lib=_abi.CHECKED_LIB_PATH)
    yield ctx
    ctx.close()


def same_results(a, b):
    """Checked against production build: identical flags, parameters within the gates."""
    assert np.array_equal(a.valid, b.valid) and np.array_equal(a.converged, b.converged)
    ok = a.valid & b.valid & (a.n_iter == b.n_iter)
    assert ok.mean() >= 0.99 * b.valid.mean()
    assert np.max(np.abs(a.y[ok] - b.y[ok]), initial=0) <= 1e-4
    assert np.max(np.abs(a.x[ok] - b.x[ok]), initial=0) <= 1e-4
    assert np.max(np.abs(a.flux[ok] / b.flux[ok] - 1), initial=0) <= 1e-5


def edge_field():
    rng = np.random.default_rng(3)
    psf = CircularGaussianPSF(fwhm=2.0)
    shape = (70, 90)
    n = 120
    ys = rng.uniform(-3, shape[0] + 3, n)
    xs = rng.uniform(-3, shape[1] + 3, n)
    fs = rng.uniform(100, 2000, n)
    img = np.zeros(shape)
    render_sources(img, psf, ys, xs, fs, model_radius=5)
    img += rng.normal(0, 1, shape)
    iv = np.ones(shape)
    iv[10:20, 30:45] = 0.0
    iv[40, :] = np.nan
    img[5, 5] = np.nan
    good = np.round(ys) >= 0
    return img, iv, psf, dict(y=ys[good], x=np.abs(xs[good]), flux=fs[good])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_edges_and_masks_checked(checked, precision):
    img, iv, psf, cat = edge_field()
    kw = dict(fixed={"fwhm": 2.0, "bkg": 0.0}, inv_var=iv, model_rad=6, max_iter=8, precision=precision)
    a = cpb.fit_all_stars_simultaneous(img, psf, cat, 4, ctx=checked, **kw)
    b = cpb.fit_all_stars_simultaneous(img, psf, cat, 4, **kw)
    same_results(a, b)
    if precision == "fp64":
        # element-wise against the CPU oracle as well: structures bit-exact, parity gates
        from oracle import orc_fit_simultaneous
        from test_gpu_sim import assert_parity
        kwd = dict(kw, debug=True)
        kwd.pop("precision")
        g = cpb.fit_all_stars_simultaneous(img, psf, cat, 4, ctx=checked, **kwd)
        o = orc_fit_simultaneous(img, psf, cat, 4, **kwd)
        assert np.array_equal(g.debug["active"], o.debug["active"])
        assert np.array_equal(g.debug["pixels"], o.debug["pixels"])
        assert_parity(g, o, tag="checked_edges")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_crowded_auto_radii_checked(checked, precision):
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(256, 256, 780, seed=1012, psf=psf, dtype=np.float32)
    kw = dict(fixed={"bkg": 0.0}, inv_var=iv, background=bkg, model_rad="auto", precision=precision,
              refine_iters=2 if precision == "mixed" else 0)
    a = cpb.fit_all_stars_simultaneous(img, psf, init, 8, ctx=checked, **kw)
    b = cpb.fit_all_stars_simultaneous(img, psf, init, 8, **kw)
    same_results(a, b)


def test_wide_boxes_checked(checked):
    """A 20 px fit radius (41 px boxes meet up to 3 x 3 regions) and a 26 px fit
    box under a 50 px model box."""
    img, bkg, iv, psf, src, init = c1_field(seed=21, n=150, shape=(160, 160))
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=20, max_iter=6)
    a = cpb.fit_all_stars_simultaneous(img, psf, init, 20, ctx=checked, **kw)
    b = cpb.fit_all_stars_simultaneous(img, psf, init, 20, **kw)
    same_results(a, b)
    sel = {k: np.asarray(v)[:10] for k, v in init.items()}
    kw = dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=50, max_iter=6)
    a = cpb.fit_all_stars_simultaneous(img, psf, sel, 26, ctx=checked, **kw)
    b = cpb.fit_all_stars_simultaneous(img, psf, sel, 26, **kw)
    same_results(a, b)
