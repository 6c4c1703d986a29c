"""Oracle matrix-free operator, LSQR and stamp bookkeeping vs dense linear algebra.

Restates test/photometry/psf_photometry_simultaneous.jl:51-216 and :455-464 with
numpy RNGs; pins the LSQR restatement against scipy's independent
Paige-Saunders implementation.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from crowdphot_b200 import CircularGaussianPSF
from oracle import (orc_apply_J, orc_apply_JT, orc_fill_stamps, orc_lsmr_dense, orc_lsqr_dense, orc_lsqr_stamp,
                    orc_morton2d, orc_ring_offsets)


def dense_J(values, pixels, npix):
    n, S2, p = values.shape
    J = np.zeros((npix, n * p))
    for a in range(n):
        for m in range(S2):
            fi = pixels[a, m]
            if fi:
                J[fi - 1, a * p:(a + 1) * p] = values[a, m]
    return J


def equilibrate(values):
    s = np.sqrt((values ** 2).sum(axis=1, keepdims=True))
    return values / np.maximum(s, np.finfo(float).eps)


def ring_pixels(n, S2, npix, step):
    return np.array([[(m + a * step) % npix + 1 for m in range(S2)] for a in range(n)], dtype=np.int32)


def test_adjoint_identity_and_dense():
    # psf_photometry_simultaneous.jl:114-151
    rng = np.random.default_rng(1234)
    p, S2, n, npix = 3, 9, 4, 20
    pixels = ring_pixels(n, S2, npix, 2)
    V = rng.standard_normal((n, S2, p))
    u, v = rng.standard_normal(npix), rng.standard_normal(n * p)
    live = np.ones(n, np.uint8)
    y = orc_apply_J(V, pixels, live, v, npix)
    z = orc_apply_JT(V, pixels, live, u)
    assert u @ y == pytest.approx(z @ v, rel=1e-12)
    J = dense_J(V, pixels, npix)
    np.testing.assert_allclose(y, J @ v, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(z, J.T @ u, rtol=1e-12, atol=1e-13)
    live[1] = 0
    Jm = J.copy()
    Jm[:, p:2 * p] = 0
    np.testing.assert_allclose(orc_apply_J(V, pixels, live, v, npix), Jm @ v, rtol=1e-12, atol=1e-13)
    z2 = orc_apply_JT(V, pixels, live, u)
    np.testing.assert_allclose(z2, Jm.T @ u, rtol=1e-12, atol=1e-13)
    assert np.all(z2[p:2 * p] == 0)


def test_masked_entries_gather_zero():
    # apply_JT!'s masked entries (pixel 0) pair with V == 0 and contribute exactly 0
    rng = np.random.default_rng(3)
    p, S2, n, npix = 3, 9, 3, 30
    pixels = ring_pixels(n, S2, npix, 5)
    pixels[1, 4] = 0
    V = rng.standard_normal((n, S2, p))
    V[1, 4] = 0
    u = rng.standard_normal(npix)
    J = dense_J(V, pixels, npix)
    np.testing.assert_allclose(orc_apply_JT(V, pixels, np.ones(n, np.uint8), u), J.T @ u, rtol=1e-12, atol=1e-13)


def test_lsqr_matches_dense_damped_normal_equations():
    # psf_photometry_simultaneous.jl:182-216
    rng = np.random.default_rng(7)
    p, S2, n = 3, 9, 6
    npix = 8 * n + 8
    pixels = ring_pixels(n, S2, npix, 8)
    V = equilibrate(rng.standard_normal((n, S2, p)))
    J = dense_J(V, pixels, npix)
    mu = 1e-3
    b = rng.standard_normal(npix)
    want = np.linalg.solve(J.T @ J + mu * np.eye(n * p), J.T @ b)
    live = np.ones(n, np.uint8)
    x, it = orc_lsqr_stamp(V, pixels, live, b, np.sqrt(mu), 200, 1e-12, 1e-12)
    # Krylov's default backward-error test (test2 <= axtol = sqrt(eps)) ends the
    # solve once ||A'r|| / (||A|| ||r||) < 1.5e-8, which bounds the relative error
    # of x by about cond(A) * sqrt(eps); the reference asserts rtol 1e-7 on its
    # own StableRNG draw, this draw (cond 9) stops at 6e-7.
    np.testing.assert_allclose(x, want, rtol=2e-6, atol=1e-9)
    live[1] = 0
    x2, _ = orc_lsqr_stamp(V, pixels, live, rng.standard_normal(npix), np.sqrt(mu), 200, 1e-12, 1e-12)
    assert np.all(x2[p:2 * p] == 0)


@pytest.mark.parametrize("damp", [0.0, 0.03, 1.0])
@pytest.mark.parametrize("itmax", [1, 3, 10])
def test_lsqr_iterates_match_scipy(damp, itmax):
    # truncated iterates agree with scipy.sparse.linalg.lsqr (Paige & Saunders 1982)
    rng = np.random.default_rng(11)
    A = rng.standard_normal((60, 12))
    b = rng.standard_normal(60)
    x, it = orc_lsqr_dense(A, b, damp, itmax, 0.0, 0.0)
    ref = spla.lsqr(A, b, damp=damp, atol=0, btol=0, conlim=0, iter_lim=itmax)
    assert it == itmax == ref[2]
    np.testing.assert_allclose(x, ref[0], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("damp", [0.0, 0.03, 1.0])
@pytest.mark.parametrize("itmax", [1, 3, 10])
def test_lsmr_iterates_match_scipy(damp, itmax):
    # solver = :lsmr: truncated iterates agree with scipy.sparse.linalg.lsmr (Fong &
    # Saunders 2011), damped and undamped
    rng = np.random.default_rng(12)
    A = rng.standard_normal((60, 12))
    b = rng.standard_normal(60)
    x, it = orc_lsmr_dense(A, b, damp, itmax, 0.0, 0.0)
    ref = spla.lsmr(A, b, damp=damp, atol=0, btol=0, conlim=0, maxiter=itmax)
    assert it == itmax == ref[2]
    np.testing.assert_allclose(x, ref[0], rtol=1e-10, atol=1e-12)


def test_lsmr_converged_solution_matches_normal_equations():
    # run to convergence with Krylov's default tolerances: the damped least-squares
    # solution (A'A + damp^2 I) x = A'b, as for lsqr
    rng = np.random.default_rng(13)
    A = rng.standard_normal((80, 10))
    b = rng.standard_normal(80)
    for damp in (0.0, 0.5):
        x, it = orc_lsmr_dense(A, b, damp, 200, 1e-12, 1e-12)
        want = np.linalg.solve(A.T @ A + damp ** 2 * np.eye(10), A.T @ b)
        assert 0 < it < 200
        np.testing.assert_allclose(x, want, rtol=1e-6, atol=1e-9)
    x, it = orc_lsmr_dense(A, np.zeros(80), 0.1, 10, 1e-6, 1e-6)
    assert it == 0 and np.all(x == 0)


def test_lsqr_zero_rhs_returns_zero():
    A = np.random.default_rng(0).standard_normal((10, 4))
    x, it = orc_lsqr_dense(A, np.zeros(10), 0.1, 10, 1e-6, 1e-6)
    assert it == 0 and np.all(x == 0)


def test_ring_offsets_prefix_boxes():
    # psf_photometry_simultaneous.jl:455-464
    R = 5
    dy, dx = orc_ring_offsets(R)
    assert len(dy) == (2 * R + 1) ** 2
    for k in range(R + 1):
        got = set(zip(dy[:(2 * k + 1) ** 2].tolist(), dx[:(2 * k + 1) ** 2].tolist()))
        assert got == {(a, b) for a in range(-k, k + 1) for b in range(-k, k + 1)}


def test_morton_interleaves_bits():
    assert orc_morton2d(0, 0) == 0
    assert orc_morton2d(1, 0) == 1
    assert orc_morton2d(0, 1) == 2
    assert orc_morton2d(3, 3) == 15
    assert orc_morton2d(2048, 1) == (1 << 22) | 2


def test_fill_preserves_frozen_columns():
    # psf_photometry_simultaneous.jl:51-112
    psf = CircularGaussianPSF(fwhm=2.0)
    fixed = {"fwhm": 2.0, "bkg": 0.0}
    R, ny, nx = 1, 30, 30
    offs = [(dy, dx) for dx in range(-R, R + 1) for dy in range(-R, R + 1)]
    ay, ax = np.array([10, 10]), np.array([10, 20])
    pixels = np.array([[(ay[a] + dy) + (ax[a] + dx - 1) * ny for (dy, dx) in offs] for a in range(2)], np.int32)
    theta = np.array([10.0, 10.0, 100.0, 10.0, 20.0, 100.0])
    w = np.ones((ny, nx))
    live = np.array([1, 0], np.uint8)
    values = np.zeros((2, 9, 3))
    colnorm = np.zeros((2, 3))
    orc_fill_stamps(psf, fixed, R, ny, nx, pixels, ay, ax, theta, w, live, values, colnorm)
    v0, c0 = values.copy(), colnorm.copy()
    assert np.all(np.isfinite(v0)) and np.all(np.isfinite(c0))
    th2 = theta.copy()
    for _ in range(5):
        th2[0] += 0.1
        orc_fill_stamps(psf, fixed, R, ny, nx, pixels, ay, ax, th2, w, live, values, colnorm)
    assert np.array_equal(values[1], v0[1]) and np.array_equal(colnorm[1], c0[1])
    assert np.all(np.isfinite(values)) and np.all(np.isfinite(colnorm))
