"""Oracle PSF arithmetic against the reference's own known answers.

Fixtures restated from test/psf/empirical_model_tests.jl:28-88 (deterministic,
no RNG), test/psf/gridded_psf_tests.jl:232-308 (finite-difference gradients)
and the analytic Gaussian.
"""
import math

import numpy as np
import pytest

from crowdphot_b200 import CircularGaussianPSF, GriddedPSFModel, ImagePSF, ArgumentError
from oracle import orc_bicubic, orc_psf_eval


def _fixture_data():
    # data = [exp(-((i - 4)^2 + (j - 4)^2) / 5) for i in 1:7, j in 1:7]
    i = np.arange(1, 8)[:, None]
    j = np.arange(1, 8)[None, :]
    return np.exp(-((i - 4.0) ** 2 + (j - 4.0) ** 2) / 5)


def test_imagepsf_known_answers():
    # empirical_model_tests.jl:31-44
    m = ImagePSF(_fixture_data(), y=11.4, x=10.3, flux=120.0, bkg=7.0, oversampling=2, normalize=True)
    assert m.data.sum() == pytest.approx(4.0)
    (ylo, yhi), (xlo, xhi) = m.extent()
    assert (ylo, yhi, xlo, xhi) == pytest.approx((9.9, 12.9, 8.8, 11.8))
    f = orc_psf_eval(m, m.y, m.x, m.flux, m.bkg, [-100.0], [-100.0], grad=False)
    assert f[0] == 7.0
    fm = ImagePSF(_fixture_data(), y=0, x=0, flux=4, bkg=1, fill_value=0.25)
    assert orc_psf_eval(fm, 0.0, 0.0, 4.0, 1.0, [-100.0], [-100.0], grad=False)[0] == 2.0


def test_imagepsf_gradient_matches_finite_differences():
    # empirical_model_tests.jl:52-69: analytic gradient vs central differences, h = 1e-5
    m = ImagePSF(_fixture_data(), y=11.4, x=10.3, flux=120.0, bkg=7.0, oversampling=2, normalize=True)
    f, g = orc_psf_eval(m, m.y, m.x, m.flux, m.bkg, [11.9], [10.8])
    f2 = orc_psf_eval(m, m.y, m.x, m.flux, m.bkg, [11.9], [10.8], grad=False)
    assert f[0] == pytest.approx(f2[0])
    p0 = np.array([m.y, m.x, m.flux])
    h = 1e-5
    for k in range(3):
        pp, pm = p0.copy(), p0.copy()
        pp[k] += h
        pm[k] -= h
        fp = orc_psf_eval(m, *pp, m.bkg, [11.9], [10.8], grad=False)[0]
        fmn = orc_psf_eval(m, *pm, m.bkg, [11.9], [10.8], grad=False)[0]
        assert g[0, k] == pytest.approx((fp - fmn) / (2 * h), rel=1e-5, abs=1e-5)


def test_bicubic_out_of_bounds_and_validation():
    # empirical_model_tests.jl:71-88
    m = ImagePSF(_fixture_data(), x=10.3, y=11.4, flux=120.0, bkg=7.0, oversampling=2, normalize=True)
    v = orc_bicubic(m.data, -1.0, 2.0, fill=0.3)[0]
    assert v[0] == 0.3 and v[1] == 0 and v[2] == 0
    with pytest.raises(ArgumentError):
        ImagePSF(np.random.rand(3, 4))
    with pytest.raises(ArgumentError):
        ImagePSF(_fixture_data(), oversampling=(2.0, 2))
    with pytest.raises(ArgumentError):
        ImagePSF(_fixture_data(), origin={"y": 4.0})
    bad = _fixture_data()
    bad[0, 0] = np.nan
    with pytest.raises(ArgumentError):
        ImagePSF(bad)


def test_bicubic_reproduces_samples_and_quadratics():
    # Keys cubic convolution is exact at the nodes and for polynomials of degree <= 2
    # away from the clamped edge stencil.
    rng = np.random.default_rng(0)
    data = rng.random((9, 11))
    for i in range(2, 8):
        for j in range(2, 10):
            v = orc_bicubic(data, float(i), float(j))[0]
            assert v[0] == pytest.approx(data[i - 1, j - 1], abs=1e-14)
    yy, xx = np.meshgrid(np.arange(1, 10), np.arange(1, 12), indexing="ij")
    q = 0.3 * yy ** 2 - 0.2 * yy * xx + 0.7 * xx ** 2 + yy - 2
    for (y, x) in [(3.25, 4.5), (5.75, 6.125), (4.0, 8.9)]:
        v = orc_bicubic(q, y, x)[0]
        assert v[0] == pytest.approx(0.3 * y ** 2 - 0.2 * y * x + 0.7 * x ** 2 + y - 2, rel=1e-12)
        assert v[1] == pytest.approx(0.6 * y - 0.2 * x + 1, rel=1e-12)
        assert v[2] == pytest.approx(-0.2 * y + 1.4 * x, rel=1e-12)


def _node(sigma2, n=15):
    c = (n + 1) / 2
    i = np.arange(1, n + 1)[:, None]
    j = np.arange(1, n + 1)[None, :]
    return ImagePSF(np.exp(-((i - c) ** 2 + (j - c) ** 2) / sigma2))


def test_gridded_four_corner_gradient_matches_finite_differences():
    # psf_fit_parity_tests.jl:459-472 node grid; gridded_psf_tests.jl:232-308 FD check
    nodes = [_node(5.0), _node(20.0), _node(20.0), _node(5.0)]
    g = GriddedPSFModel(nodes, [950.0, 950.0, 1010.0, 1010.0], [1200.0, 1275.0, 1200.0, 1275.0])
    Y, X, F = 1001.4, 1240.7, 250.0
    py = np.array([1000.0, 1001.0, 1003.0])
    px = np.array([1239.0, 1241.0, 1242.0])
    f, gr = orc_psf_eval(g, Y, X, F, 4.0, py, px)
    h = 1e-6
    for k, (dy, dx, df) in enumerate([(h, 0, 0), (0, h, 0), (0, 0, h)]):
        fp = orc_psf_eval(g, Y + dy, X + dx, F + df, 4.0, py, px, grad=False)
        fm = orc_psf_eval(g, Y - dy, X - dx, F - df, 4.0, py, px, grad=False)
        np.testing.assert_allclose(gr[:, k], (fp - fm) / (2 * h), rtol=1e-6, atol=1e-8)


def test_gaussian_value_and_gradient():
    psf = CircularGaussianPSF(fwhm=2.5)
    py, px = np.array([10.0, 11.0, 13.0]), np.array([20.0, 19.0, 22.0])
    f, g = orc_psf_eval(psf, 10.4, 20.3, 500.0, 3.0, py, px)
    gp = -4 * math.log(2)
    norm = -(math.pi * 2.5 ** 2 / gp)
    want = 500.0 / norm * np.exp(gp * ((px - 20.3) ** 2 + (py - 10.4) ** 2) / 2.5 ** 2) + 3.0
    np.testing.assert_allclose(f, want, rtol=1e-14)
    h = 1e-6
    for k, (dy, dx, df) in enumerate([(h, 0, 0), (0, h, 0), (0, 0, h)]):
        fp = orc_psf_eval(psf, 10.4 + dy, 20.3 + dx, 500.0 + df, 3.0, py, px, grad=False)
        fm = orc_psf_eval(psf, 10.4 - dy, 20.3 - dx, 500.0 - df, 3.0, py, px, grad=False)
        np.testing.assert_allclose(g[:, k], (fp - fm) / (2 * h), rtol=1e-6, atol=1e-9)


def test_gridded_constructor_validation():
    n = _node(5.0)
    with pytest.raises(ArgumentError):
        GriddedPSFModel([], [], [])
    with pytest.raises(ArgumentError):
        GriddedPSFModel([n, n, n], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0])
    with pytest.raises(ArgumentError):
        GriddedPSFModel([n, n, n, n], [0.0, 0.0, 1.0, 1.0], [0.0, 0.0, 1.0, 1.0])
