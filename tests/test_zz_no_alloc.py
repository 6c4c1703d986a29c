"""The no-allocation simultaneous fit (cpb_fit_simultaneous_device_noalloc).

It serves callers that cannot allocate device memory during a fit: hosts whose
GPU memory belongs to another allocator's pool (CUDA.jl, PyTorch), where a
cudaMalloc behind the pool's back can fail or fragment it, and loops that
cannot take cudaMalloc's implicit synchronisation.  All of its scratch lives
in a static 64 MiB device region shared by every call.  This checks, through
the C-ABI, that two calls in a row (the second one finding the first one's
data in the shared region) give the same stars as the allocating entry point
within the parity tolerances used everywhere else (1e-4 px, 1e-5 relative
flux), and that fields around the region's limit -- scalar model radii above
the fit radius and :auto radii included -- either fit or are refused with the
up-front message, never part-way through carving.  Collected last so a
failure here never hides the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-4
FLUX_TOL = 1e-5


def _device_inputs(torch, img, iv, bkg, init):
    dev = torch.device("cuda", 0)
    col = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float64).T)).to(dev)
    vec = lambda a: torch.from_numpy(np.asarray(a, np.float64)).to(dev)
    return [col(img), col(iv), col(bkg), vec(init["y"]), vec(init["x"]), vec(init["flux"])]


def _fit(ctx, fn_name, hp, P, t, ny, nx, n, S2):
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import SimOutputs
    outs = SimOutputs(n, ny, nx, S2, residual=True, debug=True)
    vp = lambda x: C.c_void_p(x.data_ptr())
    rc = getattr(ctx.lib, fn_name)(ctx.handle, hp, C.byref(P), vp(t[0]), _abi.CPB_F64, ny, nx, vp(t[1]), vp(t[2]), n,
                                   vp(t[3]), vp(t[4]), vp(t[5]), C.byref(outs.c))
    return rc, outs.result(ny, nx, S2)


def _cases():
    from crowdphot_b200 import CircularGaussianPSF
    from crowdphot_b200.simulate import add_noise, crowded_field, moffat_epsf, render_sources, simulate_sources
    rng = np.random.default_rng(2024)
    psf_g = CircularGaussianPSF(fwhm=2.5)
    src = simulate_sources((128, 128), 60, rng=rng, flux=(1e2, 1e5), flux_distribution="loguniform")
    model = np.zeros((128, 128))
    render_sources(model, psf_g, src["y"], src["x"], src["flux"], model_radius=7)
    img = add_noise(model + 100.0, rng=rng, noise="poisson")
    init = dict(y=src["y"] + rng.normal(0, 0.3, 60), x=src["x"] + rng.normal(0, 0.3, 60),
                flux=src["flux"] * rng.uniform(0.9, 1.1, 60))
    yield psf_g, img, 1.0 / (100.0 + model), np.full((128, 128), 100.0), init, 7, {"fwhm": 2.5, "bkg": 0.0}
    psf_e = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(192, 192, 440, seed=2025, psf=psf_e, dtype=np.float64)
    yield psf_e, img, iv, bkg, init, 12, {"bkg": 0.0}


def test_noalloc_matches_allocating_entry_twice():
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200.photometry import sim_params
    ctx = cpb.get_context(0)
    for psf, img, iv, bkg, init, R, fixed in _cases():
        ny, nx = img.shape
        n = len(init["y"])
        S2 = (2 * R + 1) ** 2
        hp = ctx.psf_handle(psf)
        P = sim_params(psf, R, fixed, inv_var_given=True, model_rad=R, max_iter=20)
        t = _device_inputs(torch, img, iv, bkg, init)
        rc, ref = _fit(ctx, "cpb_fit_simultaneous_device", hp, P, t, ny, nx, n, S2)
        assert rc == 0, ctx.error()
        for call in range(2):
            rc, got = _fit(ctx, "cpb_fit_simultaneous_device_noalloc", hp, P, t, ny, nx, n, S2)
            assert rc == 0, f"call {call}: {ctx.error()}"
            assert np.array_equal(got.debug["active"], ref.debug["active"])
            assert np.array_equal(got.debug["pixels"], ref.debug["pixels"])
            assert np.array_equal(got.valid, ref.valid) and np.array_equal(got.converged, ref.converged)
            ok = got.valid & ref.valid
            assert ok.sum() > 0
            assert np.max(np.abs(got.y[ok] - ref.y[ok])) <= POS_TOL
            assert np.max(np.abs(got.x[ok] - ref.x[ok])) <= POS_TOL
            assert np.max(np.abs(got.flux[ok] / ref.flux[ok] - 1)) <= FLUX_TOL
            np.testing.assert_allclose(got.flux_err[ok], ref.flux_err[ok], rtol=1e-6)
            np.testing.assert_allclose(got.residual, ref.residual, rtol=0, atol=1e-6 * np.abs(ref.residual).max())


def test_noalloc_rejects_oversized_field():
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import SimOutputs, sim_params
    from crowdphot_b200.simulate import moffat_epsf
    ctx = cpb.get_context(0)
    psf = moffat_epsf()
    ny = nx = 2048
    n = 50_000
    dev = torch.device("cuda", 0)
    img = torch.zeros((nx, ny), dtype=torch.float32, device=dev)
    ys = torch.full((n,), 100.0, dtype=torch.float64, device=dev)
    P = sim_params(psf, 12, {"bkg": 0.0}, inv_var_given=False, model_rad=12)
    outs = SimOutputs(n, ny, nx, 625, residual=False)
    vp = lambda x: C.c_void_p(x.data_ptr())
    rc = ctx.lib.cpb_fit_simultaneous_device_noalloc(ctx.handle, ctx.psf_handle(psf), C.byref(P), vp(img),
                                                     _abi.CPB_F32, ny, nx, None, None, n, vp(ys), vp(ys), vp(ys),
                                                     C.byref(outs.c))
    assert rc == _abi.CPB_ERR_ARGUMENT
    assert "too large for the no-allocation entry point" in ctx.error()


@pytest.mark.parametrize("model_rad", [12, 20, "auto"])
def test_noalloc_fields_around_the_limit_fit_or_are_refused_up_front(model_rad):
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import SimOutputs, sim_params
    from crowdphot_b200.simulate import crowded_field, moffat_epsf
    ctx = cpb.get_context(0)
    psf = moffat_epsf()
    hp = ctx.psf_handle(psf)
    seen = set()
    for side, n in ((256, 700), (384, 1500), (448, 2200), (512, 2800), (512, 3600), (640, 5000)):
        img, bkg, iv, truth, init = crowded_field(side, side, n, seed=3000 + side + n, psf=psf, dtype=np.float32)
        t = _device_inputs(torch, img, iv, bkg, init)
        P = sim_params(psf, 12, {"bkg": 0.0}, inv_var_given=True, model_rad=model_rad, max_iter=2)
        outs = SimOutputs(n, side, side, 625, residual=False)
        vp = lambda x: C.c_void_p(x.data_ptr())
        rc = ctx.lib.cpb_fit_simultaneous_device_noalloc(ctx.handle, hp, C.byref(P), vp(t[0]), _abi.CPB_F64, side,
                                                         side, vp(t[1]), vp(t[2]), n, vp(t[3]), vp(t[4]), vp(t[5]),
                                                         C.byref(outs.c))
        if rc == 0:
            seen.add("fit")
            assert outs.valid[:n].any()
        else:
            assert rc == _abi.CPB_ERR_ARGUMENT, ctx.error()
            assert "too large for the no-allocation entry point" in ctx.error(), ctx.error()
            seen.add("refused")
    assert seen == {"fit", "refused"}, seen
