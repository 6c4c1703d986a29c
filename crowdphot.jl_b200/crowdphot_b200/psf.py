"""PSF model types of the drop-in (the subset the B200 path supports).

Mirrors CrowdPhot.PSF:
  CircularGaussianPSF   src/psf/parametric_models.jl:62-115
  CircularMoffatPSF     src/psf/parametric_models.jl:672-724 (evaluation only;
                        used to tabulate empirical PSFs)
  ImagePSF              src/psf/empirical_models.jl:76-140
  GriddedPSFModel       src/psf/gridded_psf.jl:51-135

Arrays follow Julia's indexing meaning: ``data[i-1, j-1]`` is the Julia
element ``data[i, j]`` with ``i`` the row (y) and ``j`` the column (x).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GAUSS_PRE = -4.0 * math.log(2.0)


class ArgumentError(ValueError):
    """The reference's ArgumentError (invalid arguments / contract violations)."""


class AbstractPSFModel:
    """Marker base class (CrowdPhot.PSF.AbstractPSFModel)."""

    def properties(self) -> tuple[str, ...]:
        raise NotImplementedError


@dataclass
class CircularGaussianPSF(AbstractPSFModel):
    y: float = 0.0
    x: float = 0.0
    fwhm: float = 1.0
    flux: float = 1.0
    bkg: float = 0.0

    def properties(self):
        return ("y", "x", "fwhm", "flux", "bkg")

    def evaluate(self, py, px):
        """evaluate(::CircularGaussianPSF, py, px) (parametric_models.jl:79-85)."""
        dx = np.asarray(px, dtype=np.float64) - self.x
        dy = np.asarray(py, dtype=np.float64) - self.y
        sq = (dx * dx + dy * dy) / (self.fwhm * self.fwhm)
        norm = -(math.pi * self.fwhm ** 2 / GAUSS_PRE)
        return (self.flux / norm) * np.exp(GAUSS_PRE * sq) + self.bkg

    def effective_area(self):
        return math.pi * self.fwhm ** 2 / (2 * math.log(2))


@dataclass
class CircularMoffatPSF(AbstractPSFModel):
    y: float = 0.0
    x: float = 0.0
    alpha: float = 1.0
    beta: float = 3.0
    flux: float = 1.0
    bkg: float = 0.0

    def properties(self):
        return ("y", "x", "alpha", "beta", "flux", "bkg")

    def evaluate(self, py, px):
        """evaluate(::CircularMoffatPSF, py, px) (parametric_models.jl:697-701)."""
        r2 = (np.asarray(px, dtype=np.float64) - self.x) ** 2 + (np.asarray(py, dtype=np.float64) - self.y) ** 2
        amp = self.flux * (self.beta - 1) / (math.pi * self.alpha ** 2)
        return amp * (1 + r2 / self.alpha ** 2) ** (-self.beta) + self.bkg

    def effective_area(self):
        return math.pi * self.alpha ** 2 * (2 * self.beta - 1) / (self.beta - 1) ** 2


def _as_oversampling(os_):
    """_as_oversampling (empirical_models.jl:1-20): (x factor, y factor)."""
    if isinstance(os_, (int, np.integer)) and not isinstance(os_, bool):
        if os_ <= 0:
            raise ArgumentError("`oversampling` must be positive")
        return (int(os_), int(os_))
    if isinstance(os_, (tuple, list)):
        if len(os_) != 2:
            raise ArgumentError("`oversampling` must be an integer or a length-2 tuple/vector of integers")
        if not all(isinstance(v, (int, np.integer)) and not isinstance(v, bool) for v in os_):
            raise ArgumentError("length-2 `oversampling` values must be integers")
        sx, sy = int(os_[0]), int(os_[1])
        if sx <= 0 or sy <= 0:
            raise ArgumentError("`oversampling` values must be positive")
        return (sx, sy)
    raise ArgumentError("`oversampling` must be an integer or a length-2 tuple/vector of integers")


class ImagePSF(AbstractPSFModel):
    """Tabulated, oversampled empirical PSF (ImagePSF, empirical_models.jl:91-140)."""

    def __init__(self, data, *, y=0.0, x=0.0, flux=1.0, bkg=0.0, origin=None, oversampling=1, fill_value=0.0,
                 normalize=False):
        arr = np.asarray(data)
        if arr.ndim != 2:
            raise ArgumentError("`data` must be a 2D matrix")
        if not all(s >= 4 for s in arr.shape):
            raise ArgumentError("each axis of `data` must have at least 4 samples")
        if not np.all(np.isfinite(arr)):
            raise ArgumentError("all elements of `data` must be finite")
        os_ = _as_oversampling(oversampling)
        dtype = np.float32 if arr.dtype == np.float32 else np.float64
        d = np.array(arr, dtype=dtype, copy=True)
        if normalize:
            s = d.sum(dtype=np.float64)
            if not (np.isfinite(s) and s > 0):
                raise ArgumentError("cannot normalize PSF data with non-positive sum")
            d = (d * dtype(os_[0] * os_[1] / s)).astype(dtype)
        if origin is None:
            org = ((d.shape[0] + 1) / 2.0, (d.shape[1] + 1) / 2.0)
        else:
            if not isinstance(origin, dict) or set(origin.keys()) != {"y", "x"}:
                raise ArgumentError("`origin` must include exactly `y` and `x` fields")
            org = (float(origin["y"]), float(origin["x"]))
            if not (math.isfinite(org[0]) and math.isfinite(org[1])):
                raise ArgumentError("`origin` must be finite")
        self.data = d
        self.y, self.x, self.flux, self.bkg = float(y), float(x), float(flux), float(bkg)
        self.origin = {"y": org[0], "x": org[1]}
        self.oversampling = os_
        self.fill_value = float(fill_value)

    def properties(self):
        return ("y", "x", "flux", "bkg")

    def extent(self):
        ny, nx = self.data.shape
        sx, sy = self.oversampling
        oy, ox = self.origin["y"], self.origin["x"]
        return ((self.y - (oy - 1) / sy, self.y + (ny - oy) / sy), (self.x - (ox - 1) / sx, self.x + (nx - ox) / sx))

    def effective_area(self):
        denom = float(np.sum(np.asarray(self.data, dtype=np.float64) ** 2))
        return math.inf if denom == 0 else self.oversampling[0] * self.oversampling[1] / denom


class GriddedPSFModel(AbstractPSFModel):
    """Spatially varying PSF: bilinear blend of ImagePSF nodes (gridded_psf.jl:64-135)."""

    def __init__(self, psfs, grid_y, grid_x, *, y=0.0, x=0.0, flux=1.0, bkg=0.0):
        psfs = list(psfs)
        n = len(psfs)
        if n < 1:
            raise ArgumentError("`psfs` must be non-empty")
        if len(grid_y) != n or len(grid_x) != n:
            raise ArgumentError("`psfs`, `grid_y`, and `grid_x` must all have the same length")
        if not all(isinstance(p, ImagePSF) for p in psfs):
            raise ArgumentError("the B200 path supports GriddedPSFModel nodes of type ImagePSF only")
        dts = {p.data.dtype for p in psfs}
        if len(dts) != 1:
            raise ArgumentError("all `psfs` must share the same element type `T`")
        gy = np.asarray(grid_y, dtype=np.float64)
        gx = np.asarray(grid_x, dtype=np.float64)
        if not (np.all(np.isfinite(gy)) and np.all(np.isfinite(gx))):
            raise ArgumentError("`grid_y` and `grid_x` must be finite")
        if n > 1:
            uy, ux = np.unique(gy), np.unique(gx)
            if len(uy) < 2 or len(ux) < 2:
                raise ArgumentError("`grid_y` and `grid_x` must each contain at least 2 unique values unless a "
                                    "single PSF is supplied")
            if len(uy) * len(ux) != n:
                raise ArgumentError(f"`grid_y`/`grid_x` positions do not form a complete rectangular grid ({n} "
                                    f"points supplied; a {len(uy)} x {len(ux)} grid requires {len(uy) * len(ux)})")
            seen = set()
            for a, b in zip(gy, gx):
                if (a, b) in seen:
                    raise ArgumentError(f"duplicate node position at (y={a}, x={b})")
                seen.add((a, b))
        self.psfs = psfs
        self.grid_y, self.grid_x = gy, gx
        self.y, self.x, self.flux, self.bkg = float(y), float(x), float(flux), float(bkg)

    def properties(self):
        return ("y", "x", "flux", "bkg")


def replace_params(model, **kw):
    """ConstructionBase.setproperties for the fit parameters."""
    if isinstance(model, CircularGaussianPSF):
        d = dict(y=model.y, x=model.x, fwhm=model.fwhm, flux=model.flux, bkg=model.bkg)
        d.update(kw)
        return CircularGaussianPSF(**d)
    if isinstance(model, ImagePSF):
        m = ImagePSF.__new__(ImagePSF)
        m.__dict__.update(model.__dict__)
        for k, v in kw.items():
            setattr(m, k, float(v))
        return m
    if isinstance(model, GriddedPSFModel):
        m = GriddedPSFModel.__new__(GriddedPSFModel)
        m.__dict__.update(model.__dict__)
        for k, v in kw.items():
            setattr(m, k, float(v))
        return m
    raise ArgumentError(f"unsupported PSF model {type(model).__name__}")
