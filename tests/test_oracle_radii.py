"""The oracle's model_rad = :auto restatement: exact pixel / circle overlap
(apertures.jl:160-290), the unit PSF's curve of growth (curve_of_growth.jl:143-212)
and _model_radii (psf_photometry_simultaneous.jl:209-243), pinned by
known answers that do not depend on any implementation detail: the exact
overlaps of a circle tile its area, full / empty pixels weigh 1 / 0, the
weights are symmetric, and a Gaussian sampled into an ImagePSF has (nearly)
the Gaussian's analytic curve of growth and the same model radii."""
import math

import numpy as np
import pytest

from crowdphot_b200 import CircularGaussianPSF, GriddedPSFModel, ImagePSF
from oracle import (orc_aperture_weight, orc_exact_overlap, orc_model_radii_auto, orc_model_radii_auto_gaussian,
                    orc_unit_curve_of_growth)


@pytest.mark.parametrize("r", [0.3, 0.5, 0.7071, 1.0, 2.5, 3.7, 10.0, 23.4])
@pytest.mark.parametrize("centre", [(0.0, 0.0), (0.3, -0.45), (0.5, 0.5)])
def test_exact_overlaps_tile_the_circle(r, centre):
    yc, xc = centre
    R = int(math.ceil(r)) + 2
    tot = sum(orc_aperture_weight(yc, xc, r, i, j) for i in range(-R, R + 1) for j in range(-R, R + 1))
    assert tot == pytest.approx(math.pi * r * r, rel=1e-12, abs=1e-12)


def test_exact_overlap_known_values_and_symmetry():
    assert orc_exact_overlap(0.0, 0.0, 5.0) == pytest.approx(1.0)
    assert orc_exact_overlap(10.0, 0.0, 2.0) == 0.0
    assert orc_exact_overlap(0.0, 0.0, 0.5) == pytest.approx(math.pi * 0.25)  # inscribed circle
    for dx, dy in [(1.8, 0.3), (2.0, 2.0), (0.4, 1.9)]:
        a = orc_exact_overlap(dx, dy, 2.2)
        for sx, sy in [(-1, 1), (1, -1), (-1, -1)]:
            assert orc_exact_overlap(sx * dx, sy * dy, 2.2) == pytest.approx(a, rel=1e-13)
        assert orc_exact_overlap(dy, dx, 2.2) == pytest.approx(a, rel=1e-13)
        assert 0.0 < a < 1.0


def gaussian_image_psf(fwhm=2.5, os_=4, size=81):
    c = (size + 1) / 2
    off = (np.arange(1, size + 1) - c) / os_
    g = CircularGaussianPSF(fwhm=fwhm)
    data = g.evaluate(off[:, None], off[None, :])
    return GriddedPSFModel([ImagePSF(data, oversampling=os_, normalize=True)], [0.0], [0.0])


def test_image_psf_curve_of_growth_tracks_the_analytic_one():
    psf = gaussian_image_psf()
    cog = orc_unit_curve_of_growth(psf, 12)
    gcog = orc_unit_curve_of_growth(CircularGaussianPSF(fwhm=2.5), 12)
    ee, gee = cog / cog[-1], gcog / gcog[-1]
    assert np.all(np.diff(cog) >= -1e-12)
    # pixel-centre sampling of the core differs from the analytic integral by < 1 % at r >= 3
    np.testing.assert_allclose(ee[2:], gee[2:], atol=1e-2)
    np.testing.assert_allclose(ee[5:], gee[5:], atol=1e-4)


def test_model_radii_image_psf_agree_with_the_gaussian():
    psf = gaussian_image_psf()
    w = np.full(5000, 1 / 125.0)
    fl = np.geomspace(10, 1e6, 40)
    rg = orc_model_radii_auto_gaussian(2.5, 1.0, 3, 30, w, fl)
    ri = orc_model_radii_auto(psf, 1.0, 3, 30, w, fl)
    assert np.all(np.diff(ri) >= 0) and ri[0] == 3 and ri[-1] > 3
    assert np.abs(ri.astype(int) - rg).max() <= 1
