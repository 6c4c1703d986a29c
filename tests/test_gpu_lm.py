"""GPU batched fit_star (through the C-ABI) vs the oracle's fit_star, cutout by cutout."""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF, GriddedPSFModel, ImagePSF
from crowdphot_b200.simulate import flux_for_snr, moffat_epsf, psf_value
from oracle import orc_fit_star

pytestmark = pytest.mark.gpu


def cutouts(psf, n, seed, smin=9, smax=41, bkg=100.0, read_noise=5.0):
    """Isolated-star cutouts of uneven size with SNR log-uniform 5-1000."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        s = int(rng.integers(smin, smax + 1))
        y1, x1 = int(rng.integers(1, 500)), int(rng.integers(1, 500))
        yc = y1 + (s - 1) / 2 + rng.uniform(-0.5, 0.5)
        xc = x1 + (s - 1) / 2 + rng.uniform(-0.5, 0.5)
        snr = float(np.exp(rng.uniform(np.log(5), np.log(1000))))
        node = psf.psfs[0] if isinstance(psf, GriddedPSFModel) else psf
        flux = float(flux_for_snr(node, snr, background=bkg, read_noise=read_noise))
        yy, xx = np.meshgrid(np.arange(y1, y1 + s, dtype=float), np.arange(x1, x1 + s, dtype=float), indexing="ij")
        model = psf_value(psf, yc, xc, flux, yy, xx)
        img = rng.poisson(np.maximum(model + bkg, 0)).astype(float) + rng.normal(0, read_noise, model.shape) - bkg
        iv = 1.0 / (bkg + model + read_noise ** 2)
        init = (yc + rng.normal(0, 0.3), xc + rng.normal(0, 0.3), flux * rng.uniform(0.9, 1.1))
        out.append((img, iv, (y1, x1), init, (yc, xc, flux)))
    return out


@pytest.mark.parametrize("kind", ["gridded", "image", "gaussian"])
def test_lm_batch_matches_oracle(kind):
    if kind == "gaussian":
        psf = CircularGaussianPSF(fwhm=2.8)
    else:
        g = moffat_epsf()
        psf = g if kind == "gridded" else g.psfs[0]
    cs = cutouts(psf if kind != "image" else GriddedPSFModel([psf], [0.0], [0.0]), 64, seed=40)
    fixed = {"bkg": 0.0, "fwhm": 2.8} if kind == "gaussian" else {"bkg": 0.0}
    names = ("y", "x", "fwhm", "flux", "bkg") if kind == "gaussian" else ("y", "x", "flux", "bkg")

    def vec(init):
        d = dict(y=init[0], x=init[1], flux=init[2], bkg=0.0, fwhm=2.8)
        return np.array([d[k] for k in names])

    out = cpb.fit_star_batch(psf, [c[0] for c in cs], inv_vars=[c[1] for c in cs], origins=[c[2] for c in cs],
                             inits=[vec(c[3]) for c in cs], fixed=fixed)
    assert np.all(out["status"] == 0)
    for i, (img, iv, (y1, x1), init, truth) in enumerate(cs):
        s = img.shape[0]
        full = np.zeros((y1 + s - 1, x1 + s - 1))
        fiv = np.zeros_like(full)
        full[y1 - 1:, x1 - 1:] = img
        fiv[y1 - 1:, x1 - 1:] = iv
        model = cpb.replace_params(psf, **dict(zip(names, vec(init))))
        best, res = orc_fit_star(model, full, ((y1, y1 + s - 1), (x1, x1 + s - 1)), inv_var=fiv, fixed=fixed)
        assert out["iterations"][i] == res.iterations
        assert bool(out["converged"][i]) == res.converged
        p = out["params"][i]
        assert abs(p[0] - best.y) < 1e-7 and abs(p[1] - best.x) < 1e-7
        k = names.index("flux")
        assert abs(p[k] / best.flux - 1) < 1e-9
        np.testing.assert_allclose(out["cov"][i], res.cov, rtol=1e-6, atol=1e-12)
        assert out["cost"][i] == pytest.approx(res.minimum, rel=1e-9)


def test_fit_star_four_corner_gridded_truth():
    c = 8.0
    i = np.arange(1, 16)[:, None]
    j = np.arange(1, 16)[None, :]
    mk = lambda s2: ImagePSF(np.exp(-((i - c) ** 2 + (j - c) ** 2) / s2))
    g = GriddedPSFModel([mk(5.0), mk(20.0), mk(20.0), mk(5.0)], [950.0, 950.0, 1010.0, 1010.0],
                        [1200.0, 1275.0, 1200.0, 1275.0], y=1000.9, x=1241.2, flux=230.0, bkg=4.4)
    from oracle import orc_psf_eval
    yy, xx = np.meshgrid(np.arange(991, 1011), np.arange(1231, 1251), indexing="ij")
    f = orc_psf_eval(g, 1001.4, 1240.7, 250.0, 4.0, yy.ravel().astype(float), xx.ravel().astype(float), grad=False)
    img = np.zeros((1010, 1250))
    img[990:1010, 1230:1250] = f.reshape(yy.shape)
    best, res = cpb.fit_star(g, img, ((991, 1010), (1231, 1250)), inv_var=np.ones_like(img), x_tol=1e-7,
                             max_iter=100)
    assert res.converged
    assert best.y == pytest.approx(1001.4, abs=1e-7) and best.x == pytest.approx(1240.7, abs=1e-7)
    assert best.flux == pytest.approx(250.0, rel=1e-7) and best.bkg == pytest.approx(4.0, abs=1e-6)


def test_fit_star_errors():
    m = CircularGaussianPSF(y=8.0, x=8.0, fwhm=2.0, flux=400.0, bkg=3.0)
    img = np.ones((15, 15))
    with pytest.raises(ArgumentError, match="too few valid"):
        cpb.fit_star(m, img, inv_var=np.zeros_like(img))
    with pytest.raises(ArgumentError, match="all model parameters are fixed"):
        cpb.fit_star(m, img, fixed=dict(y=1, x=1, fwhm=1, flux=1, bkg=1))


def test_packed_cutouts_host_and_device_entries_match_oracle():
    """The C4 cutout workload (isolated stars, sides 9..41, SNR 5..1000, float32
    pixels): host-buffer entry, device-buffer entry and the oracle agree cutout by cutout.
    12,000 cutouts are 69 MB of pixels and weights, so the host entry uploads them
    in two chunks that overlap the fits."""
    import torch
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import _lm_outputs, _lm_result_struct, lm_params
    from crowdphot_b200.simulate import lm_cutouts
    from oracle.ffi import orc_fit_star_packed
    psf = moffat_epsf()
    d = lm_cutouts(12000, seed=41)
    args = (d["pix"], d["offsets"], d["ny"], d["nx"], d["y1"], d["x1"], d["init"])
    fixed = {"bkg": 0.0}
    host = cpb.fit_star_packed(psf, *args, inv_var=d["inv_var"], fixed=fixed)
    ref, _ = orc_fit_star_packed(psf, *args, inv_var=d["inv_var"], fixed=fixed, threads=0)
    assert np.all(host["status"] == 0) and np.all(ref["status"] == 0)
    assert np.array_equal(host["iterations"], ref["iterations"])
    assert np.array_equal(host["converged"], ref["converged"])
    assert np.max(np.abs(host["params"][:, :2] - ref["params"][:, :2])) < 1e-7
    assert np.max(np.abs(host["params"][:, 2] / ref["params"][:, 2] - 1)) < 1e-9
    np.testing.assert_allclose(host["cov"], ref["cov"], rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(host["cost"], ref["cost"], rtol=1e-9)

    ctx = cpb.get_context(0)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dpix, div, doff = t(d["pix"]), t(d["inv_var"]), t(d["offsets"])
    dny, dnx, dy1, dx1, dinit = t(d["ny"]), t(d["nx"]), t(d["y1"]), t(d["x1"]), t(d["init"])
    outs = {k: torch.from_numpy(v).to(dev) for k, v in _lm_outputs(len(d["ny"]), 4, 3).items()}
    r = _lm_result_struct(outs, lambda a: a.data_ptr())
    P = lm_params(psf, fixed)
    vp = lambda a: a.data_ptr()
    rc = ctx.lib.cpb_fit_lm_batch_device(ctx.handle, ctx.psf_handle(psf), P, len(d["ny"]), vp(doff), vp(dny),
                                         vp(dnx), vp(dy1), vp(dx1), vp(dpix), _abi.CPB_F32, vp(div), vp(dinit),
                                         d["pix"].size, r)
    assert rc == 0, ctx.error()
    assert r.device_seconds > 0
    for k in ("params", "cov", "cost", "chisq", "iterations", "converged", "status"):
        assert np.array_equal(outs[k].cpu().numpy(), host[k]), k
