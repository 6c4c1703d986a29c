"""Serving (cpb_server_*): continuous batching of fit_all_stars_simultaneous
requests on one GPU, through the C-ABI.

The gates: every request's result equals the same request fitted alone
(bit-identical: the fits are deterministic and requests share no device state);
requests submitted together run overlapped; admission by device memory
serialises requests that do not fit together and refuses one that never fits;
queued requests can be cancelled; argument errors come back per request.
"""
import numpy as np
import pytest

import crowdphot_b200 as cpb
from crowdphot_b200 import ArgumentError, CircularGaussianPSF
from crowdphot_b200.simulate import crowded_field, moffat_epsf

pytestmark = pytest.mark.gpu

KW = dict(fixed={"bkg": 0.0}, model_rad=12)


def fields():
    psf = moffat_epsf()
    out = []
    for i, (ny, nx, n) in enumerate([(96, 96, 40), (160, 128, 120), (256, 256, 700), (128, 200, 200),
                                     (200, 200, 500), (300, 260, 1000)]):
        img, bkg, iv, truth, init = crowded_field(ny, nx, n, seed=5000 + i, psf=psf, dtype=np.float32)
        out.append((img, bkg, iv, init))
    return psf, out


def assert_same(a, b):
    for k in ("y", "x", "flux", "y_err", "x_err", "flux_err", "n_iter", "converged", "valid", "chisq"):
        assert np.array_equal(getattr(a, k), getattr(b, k), equal_nan=True), k
    assert a.n_passes == b.n_passes and a.n_failed == b.n_failed


def test_served_results_equal_alone_and_overlap():
    psf, fl = fields()
    with cpb.Server(max_inflight=3) as sv:
        reqs = []
        for i, (img, bkg, iv, init) in enumerate(fl):
            prec = "mixed" if i == 4 else "fp64"
            reqs.append((sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, precision=prec, **KW), prec))
        served = [(r.result(timeout=300), prec) for r, prec in reqs]
        infos = [r.poll() for r, _ in reqs]
    for (img, bkg, iv, init), (res, prec) in zip(fl, served):
        alone = cpb.fit_all_stars_simultaneous(img, psf, init, 12, inv_var=iv, background=bkg, precision=prec,
                                               residual=False, **KW)
        assert_same(res, alone)
    assert all(i["state"] == "done" and i["status"] == 0 for i in infos)
    assert len({i["slot"] for i in infos}) > 1
    # at least two requests ran at the same time
    spans = sorted((i["start_time"], i["end_time"]) for i in infos)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1)), spans


def test_admission_by_device_memory():
    psf, fl = fields()
    img, bkg, iv, init = fl[5]
    import torch
    free, total = torch.cuda.mem_get_info()
    # learn this request's estimate, then give a server room for one such fit at a time
    with cpb.Server(max_inflight=2) as sv:
        est = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW).wait(timeout=300)["est_bytes"]
    free, total = torch.cuda.mem_get_info()
    reserve = int(free - 1.5 * est)
    with cpb.Server(max_inflight=2, hbm_reserve_bytes=reserve) as sv:
        a = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        b = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        ia, ib = a.wait(timeout=300), b.wait(timeout=300)
        assert ia["state"] == ib["state"] == "done"
        first, second = sorted([ia, ib], key=lambda i: i["start_time"])
        assert second["start_time"] >= first["end_time"] - 1e-3, (ia, ib)
        assert_same(a.result(), b.result())
    # a request larger than the whole budget is refused, not run
    with cpb.Server(max_inflight=1, hbm_reserve_bytes=int(free)) as sv:
        r = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        info = r.wait(timeout=60)
        assert info["state"] == "failed" and info["status"] == -3 and "admission refused" in info["error"]
        with pytest.raises(cpb.CudaError, match="admission refused"):
            r.result()


def test_cancel_poll_and_errors():
    psf, fl = fields()
    gpsf = CircularGaussianPSF(fwhm=2.0)
    with cpb.Server(max_inflight=1) as sv:
        img, bkg, iv, init = fl[5]
        r1 = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        r2 = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        r3 = sv.submit(img, psf, init, 12, inv_var=iv, background=bkg, **KW)
        assert r3.poll()["state"] in ("queued", "running")
        cancelled = r3.cancel()
        bad = sv.submit(np.zeros((32, 32)), gpsf, dict(y=[16.0], x=[16.0], flux=[100.0]), 5,
                        fixed={"fwhm": 2.0, "bkg": 0.0}, damping="levenberg", model_rad=5)
        assert r1.wait(timeout=300)["state"] == "done"
        assert r2.wait(timeout=300)["state"] == "done"
        if cancelled:
            assert r3.wait(timeout=10)["state"] == "cancelled"
            with pytest.raises(RuntimeError, match="cancelled"):
                r3.result()
        with pytest.raises(ArgumentError, match="LevenbergDamping"):
            bad.result(timeout=60)
        assert bad.poll()["state"] == "failed"
