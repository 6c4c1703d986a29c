"""Synthetic crowded fields (restating CrowdPhot's simulation.jl with numpy RNGs).

The reference draws with StableRNGs streams that cannot be reproduced here,
so images are not bit-identical to the reference's fixtures; the
distributions are the same:
  _sample_flux          src/simulation.jl:1-28 (uniform / loguniform / powerlaw)
  flux_for_snr          src/simulation.jl:59-80
  simulate_sources      src/simulation.jl:211-281 (uniform placement, min_separation)
  render_sources!       src/simulation.jl:300-347 (bounding box from extent or model_radius)
  add_noise!            src/simulation.jl:409-435 (Poisson with gain, Gaussian read noise)
Rendering evaluates the same PSF models the fitter uses (numpy restatement
of the bicubic ePSF and the circular Gaussian), so noiseless fits recover
the truth to rounding.
"""
from __future__ import annotations

import math

import numpy as np

from .psf import ArgumentError, CircularGaussianPSF, CircularMoffatPSF, GriddedPSFModel, ImagePSF, GAUSS_PRE


def sample_flux(rng, flux, distribution="uniform", power=2.0, size=None):
    if np.isscalar(flux):
        return np.full(size, float(flux)) if size is not None else float(flux)
    lo, hi = float(flux[0]), float(flux[1])
    if not (lo > 0 and hi >= lo):
        raise ArgumentError("flux range must be positive and ordered")
    u = rng.random(size)
    if distribution == "uniform":
        return lo + u * (hi - lo)
    if distribution == "loguniform" or (distribution == "powerlaw" and abs(power - 1) < 1e-15):
        return np.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))
    if distribution == "powerlaw":
        q = 1 - float(power)
        return (lo ** q + u * (hi ** q - lo ** q)) ** (1 / q)
    raise ArgumentError(f"unsupported flux distribution `{distribution}`")


def flux_for_snr(model, snr, *, background, read_noise=0.0, gain=1.0):
    """flux_for_snr (simulation.jl:59-80)."""
    snr = np.asarray(snr, dtype=np.float64)
    s2b = background / gain + read_noise ** 2
    bv = model.effective_area() * s2b
    t = snr ** 2 / gain
    return (t + np.sqrt(t ** 2 + 4 * snr ** 2 * bv)) / 2


def simulate_sources(shape, n, *, rng, flux=(100.0, 1000.0), flux_distribution="uniform", flux_power=2.0,
                     min_separation=0.0, border=0):
    """Uniform positions in the border-trimmed image (simulation.jl:211-281)."""
    by, bx = (border, border) if np.isscalar(border) else border
    ymin, ymax = 1 + by, shape[0] - by
    xmin, xmax = 1 + bx, shape[1] - bx
    if not (xmin <= xmax and ymin <= ymax):
        raise ArgumentError("border leaves no valid source-placement area")
    if min_separation <= 0:
        x = xmin + rng.random(n) * (xmax - xmin)
        y = ymin + rng.random(n) * (ymax - ymin)
        f = sample_flux(rng, flux, flux_distribution, flux_power, size=n)
        return dict(y=y, x=x, flux=np.asarray(f, dtype=np.float64))
    ys, xs, fs = [], [], []
    cell = float(min_separation)
    grid: dict = {}
    attempts = 0
    max_attempts = max(10_000, 200 * n)
    while len(ys) < n and attempts < max_attempts:
        attempts += 1
        x = xmin + rng.random() * (xmax - xmin)
        y = ymin + rng.random() * (ymax - ymin)
        cy, cx = int((y - ymin) // cell), int((x - xmin) // cell)
        ok = True
        for iy in (cy - 1, cy, cy + 1):
            for ix in (cx - 1, cx, cx + 1):
                for k in grid.get((iy, ix), ()):
                    if (y - ys[k]) ** 2 + (x - xs[k]) ** 2 < min_separation ** 2:
                        ok = False
        if not ok:
            continue
        grid.setdefault((cy, cx), []).append(len(ys))
        ys.append(y)
        xs.append(x)
        fs.append(float(sample_flux(rng, flux, flux_distribution, flux_power)))
    return dict(y=np.array(ys), x=np.array(xs), flux=np.array(fs))


def _cubic_rows(d, ly, lx, du, ny, nx):
    """Row values / derivatives of the clamped 4x4 stencil (empirical_models.jl:270-285)."""
    ix = [np.clip(lx - 1, 1, nx), lx, lx + 1, np.clip(lx + 2, 1, nx)]
    iy = [np.clip(ly - 1, 1, ny), ly, ly + 1, np.clip(ly + 2, 1, ny)]
    rows, drows = [], []
    for r in range(4):
        a, b, c, e = (d[iy[r] - 1, ix[k] - 1] for k in range(4))
        k1 = (c - a) / 2
        k4 = c - b - k1
        k2 = 3 * k4 - (e - b) / 2 + k1
        k3 = k4 - k2
        rows.append(du * (du * (du * k3 + k2) + k1) + b)
        drows.append(du * (3 * du * k3 + 2 * k2) + k1)
    return rows, drows


def image_psf_eval(node: ImagePSF, Y, X, py, px):
    """Unit-flux ePSF value at detector pixels (py, px) for a star at (Y, X), vectorised."""
    d = np.asarray(node.data, dtype=np.float64)
    ny, nx = d.shape
    sx, sy = node.oversampling
    u = sx * (px - X) + node.origin["x"]
    v = sy * (py - Y) + node.origin["y"]
    inb = np.isfinite(u) & np.isfinite(v) & (u >= 1) & (u <= nx) & (v >= 1) & (v <= ny)
    uc = np.where(inb, u, 1.0)
    vc = np.where(inb, v, 1.0)
    lx = np.clip(np.floor(uc).astype(np.int64), 1, nx - 1)
    ly = np.clip(np.floor(vc).astype(np.int64), 1, ny - 1)
    du = uc - lx
    dv = vc - ly
    rows, _ = _cubic_rows(d, ly, lx, du, ny, nx)
    v1 = (rows[2] - rows[0]) / 2
    v4 = rows[2] - rows[1] - v1
    v2 = 3 * v4 - (rows[3] - rows[1]) / 2 + v1
    v3 = v4 - v2
    val = dv * (dv * (dv * v3 + v2) + v1) + rows[1]
    return np.where(inb, val, node.fill_value)


def psf_value(psf, Y, X, flux, py, px):
    """flux * unit profile at (py, px) for stars at (Y, X) (broadcasting)."""
    if isinstance(psf, CircularGaussianPSF):
        sq = ((px - X) ** 2 + (py - Y) ** 2) / psf.fwhm ** 2
        norm = -(math.pi * psf.fwhm ** 2 / GAUSS_PRE)
        return (flux / norm) * np.exp(GAUSS_PRE * sq)
    if isinstance(psf, CircularMoffatPSF):
        r2 = (px - X) ** 2 + (py - Y) ** 2
        amp = flux * (psf.beta - 1) / (math.pi * psf.alpha ** 2)
        return amp * (1 + r2 / psf.alpha ** 2) ** (-psf.beta)
    if isinstance(psf, ImagePSF):
        return flux * image_psf_eval(psf, Y, X, py, px)
    if isinstance(psf, GriddedPSFModel):
        if len(psf.psfs) != 1:
            raise ArgumentError("simulation renders single-node GriddedPSFModel only")
        return flux * image_psf_eval(psf.psfs[0], Y, X, py, px)
    raise ArgumentError(f"unsupported PSF {type(psf).__name__}")


def psf_half_extent(psf):
    if isinstance(psf, (ImagePSF, GriddedPSFModel)):
        nd = psf if isinstance(psf, ImagePSF) else psf.psfs[0]
        (ylo, yhi), (xlo, xhi) = nd.extent()
        return max(-ylo, yhi, -xlo, xhi)
    if isinstance(psf, CircularGaussianPSF):
        return 5 * psf.fwhm
    return 10.0


def render_sources(image, psf, ys, xs, fs, *, model_radius=None, chunk=1024):
    """Adds each source's model to `image` (render_sources!, simulation.jl:321-347)."""
    ny, nx = image.shape
    rad = psf_half_extent(psf) if model_radius is None else float(model_radius)
    H = int(math.ceil(rad)) + 2
    offs = np.arange(-H, H + 1)
    for s in range(0, len(ys), chunk):
        Y = np.asarray(ys[s:s + chunk], dtype=np.float64)
        X = np.asarray(xs[s:s + chunk], dtype=np.float64)
        F = np.asarray(fs[s:s + chunk], dtype=np.float64)
        ylo = np.maximum(1, np.floor(Y - rad)).astype(np.int64)
        yhi = np.minimum(ny, np.ceil(Y + rad)).astype(np.int64)
        xlo = np.maximum(1, np.floor(X - rad)).astype(np.int64)
        xhi = np.minimum(nx, np.ceil(X + rad)).astype(np.int64)
        cy = np.round(Y).astype(np.int64)
        cx = np.round(X).astype(np.int64)
        gy = cy[:, None, None] + offs[None, :, None]
        gx = cx[:, None, None] + offs[None, None, :]
        gy, gx = np.broadcast_arrays(gy, gx)
        keep = (gy >= ylo[:, None, None]) & (gy <= yhi[:, None, None]) & (gx >= xlo[:, None, None]) & \
               (gx <= xhi[:, None, None])
        vals = psf_value(psf, Y[:, None, None], X[:, None, None], F[:, None, None], gy.astype(np.float64),
                         gx.astype(np.float64))
        gyk, gxk, vk = gy[keep], gx[keep], vals[keep]
        np.add.at(image, (gyk - 1, gxk - 1), vk)
    return image


def add_noise(image, *, rng, noise="poisson_gaussian", read_noise=0.0, gain=1.0):
    """add_noise! (simulation.jl:409-435)."""
    if noise in (None, "none"):
        return image
    if noise in ("poisson", "poisson_gaussian"):
        lam = np.maximum(0.0, image * gain)
        image[...] = rng.poisson(lam) / gain
    if noise in ("gaussian", "poisson_gaussian"):
        image += read_noise * rng.standard_normal(image.shape)
    return image


def moffat_epsf(fwhm=2.8, beta=3.0, oversampling=4, size=101, dtype=np.float64):
    """Tabulated ePSF of a CircularMoffatPSF on an oversampled grid (node samples at
    (i - origin)/oversampling px), normalised to sum = oversampling^2."""
    alpha = fwhm / (2 * math.sqrt(2 ** (1 / beta) - 1))
    c = (size + 1) / 2
    off = (np.arange(1, size + 1) - c) / oversampling
    m = CircularMoffatPSF(0.0, 0.0, alpha, beta, 1.0, 0.0)
    data = m.evaluate(off[:, None], off[None, :])
    node = ImagePSF(data.astype(dtype), oversampling=oversampling, normalize=True)
    return GriddedPSFModel([node], [0.0], [0.0])


def crowded_field(ny, nx, n, *, seed, psf=None, flux=(1e1, 1e6), flux_distribution="powerlaw", flux_power=1.5,
                  read_noise=5.0, gain=1.0, bkg_lo=50.0, bkg_span=150.0, dtype=np.float32, border=0,
                  init_sigma=0.3, init_flux=(0.9, 1.1), model_radius=None):
    """The 2048^2 crowded-field workload (any size): power-law fluxes, a smooth
    background 50 + 150 (0.6 u + 0.4 v^2) in [50, 200], Poisson + Gaussian
    noise, inverse-variance weights 1/(bkg + model + read_noise^2) and
    perturbed initial guesses.  Returns (image, background, inv_var, truth, init)."""
    rng = np.random.default_rng(seed)
    psf = psf if psf is not None else moffat_epsf()
    src = simulate_sources((ny, nx), n, rng=rng, flux=flux, flux_distribution=flux_distribution,
                           flux_power=flux_power, border=border)
    model = np.zeros((ny, nx), dtype=np.float64)
    render_sources(model, psf, src["y"], src["x"], src["flux"], model_radius=model_radius)
    u = (np.arange(1, nx + 1) - 1) / max(nx - 1, 1)
    v = (np.arange(1, ny + 1) - 1) / max(ny - 1, 1)
    bkg = bkg_lo + bkg_span * (0.6 * u[None, :] + 0.4 * (v ** 2)[:, None])
    img = add_noise(bkg + model, rng=rng, noise="poisson_gaussian", read_noise=read_noise, gain=gain)
    inv_var = 1.0 / (bkg + model + read_noise ** 2)
    init = dict(y=src["y"] + rng.normal(0, init_sigma, src["y"].size),
                x=src["x"] + rng.normal(0, init_sigma, src["x"].size),
                flux=src["flux"] * rng.uniform(init_flux[0], init_flux[1], src["flux"].size))
    return img.astype(dtype), bkg.astype(dtype), inv_var.astype(dtype), src, init


def _catmull_rom(t):
    """The four stencil weights of the clamped cubic in _cubic_rows, as functions of the fraction t."""
    t2, t3 = t * t, t * t * t
    return np.stack([(-t3 + 2 * t2 - t) / 2, (3 * t3 - 5 * t2 + 2) / 2, (-3 * t3 + 4 * t2 + t) / 2, (t3 - t2) / 2],
                    axis=-1)


def _axis_stencil(Yc, first, side, os_, origin, n):
    """Per-cutout stencil of one axis for pixels first..first+side-1 of a star at Yc: the
    grid fraction is the same on every pixel (the oversampling is an integer), so one weight
    vector serves the whole axis.  Returns (indices (k, side, 4), in-grid mask (k, side), weights (k, 4))."""
    v = os_ * (first[:, None] + np.arange(side)[None, :] - Yc[:, None]) + origin
    inb = (v >= 1) & (v <= n)
    lv = np.floor(np.where(inb, v, 1.0)).astype(np.int64)
    t = v[:, 0] - np.floor(v[:, 0])
    idx = np.clip(np.stack([lv - 1, lv, lv + 1, lv + 2], axis=-1), 1, n) - 1
    return idx, inb, _catmull_rom(t)


def render_cutouts(node: ImagePSF, Yc, Xc, flux, y1, x1, side):
    """flux * ePSF over square cutouts of one side (k, side, side), separably: rows are
    contracted first over the grid's columns, then the column stencil is applied."""
    d = np.asarray(node.data, dtype=np.float64)
    ny, nx = d.shape
    sx, sy = node.oversampling
    iy, my, wy = _axis_stencil(Yc, y1, side, sy, node.origin["y"], ny)
    ix, mx, wx = _axis_stencil(Xc, x1, side, sx, node.origin["x"], nx)
    rows = np.einsum("kr,kirc->kic", wy, d[iy])                     # (k, side, nx)
    k = np.arange(len(Yc))[:, None, None, None]
    g = rows[k, np.arange(side)[None, :, None, None], ix[:, None, :, :]]  # (k, side_i, side_j, 4)
    val = np.einsum("kc,kijc->kij", wx, g)
    val = np.where(my[:, :, None] & mx[:, None, :], val, node.fill_value)
    return flux[:, None, None] * val


def lm_cutouts(n, *, seed, psf=None, smin=9, smax=41, snr=(5.0, 1000.0), bkg=100.0, read_noise=5.0, gain=1.0,
               dtype=np.float32, init_sigma=0.3, init_flux=(0.9, 1.1)):
    """Isolated-star cutouts of uneven size for batched fit_star: side ~ U{smin..smax},
    star at the cutout centre + U(-0.5, 0.5) px, flux from an SNR drawn log-uniform
    in `snr` via flux_for_snr (bkg 100, read noise 5, gain 1), Poisson + Gaussian
    noise, background subtracted, inverse-variance weights.  Cutouts are returned
    concatenated (column-major each) with offsets, sizes and 1-based origins."""
    rng = np.random.default_rng(seed)
    psf = psf if psf is not None else moffat_epsf()
    node = psf.psfs[0] if isinstance(psf, GriddedPSFModel) else psf
    sides = rng.integers(smin, smax + 1, n)
    y1 = rng.integers(1, 4000, n)
    x1 = rng.integers(1, 4000, n)
    yc = y1 + (sides - 1) / 2 + rng.uniform(-0.5, 0.5, n)
    xc = x1 + (sides - 1) / 2 + rng.uniform(-0.5, 0.5, n)
    s = np.exp(rng.uniform(np.log(snr[0]), np.log(snr[1]), n))
    flux = flux_for_snr(node, s, background=bkg, read_noise=read_noise, gain=gain)
    sizes = sides.astype(np.int64) ** 2
    offsets = np.zeros(n, np.int64)
    offsets[1:] = np.cumsum(sizes)[:-1]
    pix = np.empty(int(sizes.sum()), dtype=dtype)
    iv = np.empty_like(pix)
    for side in np.unique(sides):
        idx = np.nonzero(sides == side)[0]
        model = render_cutouts(node, yc[idx], xc[idx], flux[idx], y1[idx], x1[idx], int(side))
        img = rng.poisson(np.maximum(model + bkg, 0) * gain) / gain + read_noise * rng.standard_normal(model.shape)
        var = bkg + model + read_noise ** 2
        # column-major per cutout: (k, i, j) -> transpose to (k, j, i) then flatten
        flat_img = np.ascontiguousarray(np.transpose(img - bkg, (0, 2, 1))).reshape(len(idx), -1)
        flat_iv = np.ascontiguousarray(np.transpose(1.0 / var, (0, 2, 1))).reshape(len(idx), -1)
        at = offsets[idx, None] + np.arange(side * side)[None, :]
        pix[at] = flat_img
        iv[at] = flat_iv
    init = np.stack([yc + rng.normal(0, init_sigma, n), xc + rng.normal(0, init_sigma, n),
                     flux * rng.uniform(init_flux[0], init_flux[1], n), np.zeros(n)], axis=1)
    return dict(pix=pix, inv_var=iv, offsets=offsets, ny=sides.astype(np.int32), nx=sides.astype(np.int32),
                y1=y1.astype(np.int32), x1=x1.astype(np.int32), init=init, truth=np.stack([yc, xc, flux], 1))


def lm_groups(n, *, seed, psf=None, kmin=2, kmax=12, snr=(5.0, 1000.0), bkg=100.0, read_noise=5.0, gain=1.0,
              dtype=np.float32, init_sigma=0.3, init_flux=(0.9, 1.1), chunk=8192):
    """Blended groups for the batched simultaneous fit: group g holds k ~ U{kmin..kmax}
    stars placed uniformly in a (8k + 17)^2 cutout, fluxes from an SNR drawn log-uniform
    in `snr` via flux_for_snr (bkg 100, read noise 5, gain 1), Poisson + Gaussian noise,
    background subtracted, inverse-variance weights, perturbed initial guesses.  Groups
    are packed like lm_cutouts (column-major each, offsets, sides) with star offsets
    into the concatenated catalogue (coordinates local to each group, 1-based)."""
    rng = np.random.default_rng(seed)
    psf = psf if psf is not None else moffat_epsf()
    node = psf.psfs[0] if isinstance(psf, GriddedPSFModel) else psf
    k = rng.integers(kmin, kmax + 1, n)
    side = (8 * k + 17).astype(np.int64)
    sizes = side * side
    offsets = np.zeros(n, np.int64)
    offsets[1:] = np.cumsum(sizes)[:-1]
    star_off = np.zeros(n + 1, np.int64)
    star_off[1:] = np.cumsum(k)
    ns = int(star_off[-1])
    grp = np.repeat(np.arange(n), k)
    sg = side[grp].astype(np.float64)
    ys = rng.uniform(1.0, sg)
    xs = rng.uniform(1.0, sg)
    s = np.exp(rng.uniform(np.log(snr[0]), np.log(snr[1]), ns))
    flux = flux_for_snr(node, s, background=bkg, read_noise=read_noise, gain=gain)
    model = np.zeros(int(sizes.sum()), np.float64)
    H = 13
    box = 2 * H + 1
    for c0 in range(0, ns, chunk):
        sl = slice(c0, min(c0 + chunk, ns))
        cy = np.round(ys[sl]).astype(np.int64)
        cx = np.round(xs[sl]).astype(np.int64)
        val = render_cutouts(node, ys[sl], xs[sl], flux[sl], cy - H, cx - H, box)  # (m, box, box)
        gy = (cy - H)[:, None, None] + np.arange(box)[None, :, None]
        gx = (cx - H)[:, None, None] + np.arange(box)[None, None, :]
        gy, gx = np.broadcast_arrays(gy, gx)
        sd = side[grp[sl]][:, None, None]
        keep = (gy >= 1) & (gy <= sd) & (gx >= 1) & (gx <= sd)
        flat = offsets[grp[sl]][:, None, None] + (gy - 1) + (gx - 1) * sd
        np.add.at(model, flat[keep], val[keep])
    img = rng.poisson(np.maximum(model + bkg, 0) * gain) / gain + read_noise * rng.standard_normal(model.size)
    pix = (img - bkg).astype(dtype)
    iv = (1.0 / (bkg + model + read_noise ** 2)).astype(dtype)
    init_y = ys + rng.normal(0, init_sigma, ns)
    init_x = xs + rng.normal(0, init_sigma, ns)
    init_f = flux * rng.uniform(init_flux[0], init_flux[1], ns)
    return dict(pix=pix, inv_var=iv, offsets=offsets, ny=side.astype(np.int32), nx=side.astype(np.int32),
                star_offsets=star_off, y=init_y, x=init_x, flux=init_f, truth=np.stack([ys, xs, flux], 1))


def served_field(side, density, *, seed, psf=None, flux=(1e1, 1e6), flux_power=1.5, read_noise=5.0, gain=1.0,
                 bkg_lo=50.0, bkg_span=150.0, dtype=np.float32, init_sigma=0.3, init_flux=(0.9, 1.1), chunk=16384):
    """One field of a served request stream: side x side pixels, density * side^2
    stars placed uniformly, power-law fluxes, the crowded-field background and
    noise model, rendered per star over a +-13 px box with the separable ePSF
    stencil (single-node image PSFs).  Returns (image, background, inv_var, truth, init)."""
    rng = np.random.default_rng(seed)
    psf = psf if psf is not None else moffat_epsf()
    node = psf.psfs[0] if isinstance(psf, GriddedPSFModel) else psf
    n = int(round(density * side * side))
    src = simulate_sources((side, side), n, rng=rng, flux=flux, flux_distribution="powerlaw", flux_power=flux_power)
    ys, xs, fs = (np.asarray(src[k], np.float64) for k in ("y", "x", "flux"))
    model = np.zeros(side * side, np.float64)
    H = 13
    box = 2 * H + 1
    for c0 in range(0, n, chunk):
        sl = slice(c0, min(c0 + chunk, n))
        cy = np.round(ys[sl]).astype(np.int64)
        cx = np.round(xs[sl]).astype(np.int64)
        val = render_cutouts(node, ys[sl], xs[sl], fs[sl], cy - H, cx - H, box)
        gy = (cy - H)[:, None, None] + np.arange(box)[None, :, None]
        gx = (cx - H)[:, None, None] + np.arange(box)[None, None, :]
        gy, gx = np.broadcast_arrays(gy, gx)
        keep = (gy >= 1) & (gy <= side) & (gx >= 1) & (gx <= side)
        np.add.at(model, ((gy - 1) * side + (gx - 1))[keep], val[keep])  # row-major (y, x)
    model = model.reshape(side, side)
    u = (np.arange(1, side + 1) - 1) / max(side - 1, 1)
    bkg = bkg_lo + bkg_span * (0.6 * u[None, :] + 0.4 * (u ** 2)[:, None])
    img = rng.poisson(np.maximum(bkg + model, 0) * gain) / gain + read_noise * rng.standard_normal(model.shape)
    inv_var = 1.0 / (bkg + model + read_noise ** 2)
    init = dict(y=ys + rng.normal(0, init_sigma, n), x=xs + rng.normal(0, init_sigma, n),
                flux=fs * rng.uniform(init_flux[0], init_flux[1], n))
    return img.astype(dtype), bkg.astype(dtype), inv_var.astype(dtype), src, init


def c1_field(seed=1001, n=200, shape=(256, 256)):
    """The plain CPU-runnable configuration: a Float64 image with n stars at
    uniform sub-pixel positions, fluxes log-uniform 1e2-1e5, a CircularGaussianPSF
    of FWHM 2.5 (15 x 15 boxes), flat background 100 + Poisson noise and
    inverse-variance weights; initial guesses perturbed by N(0, 0.3 px) in y / x and
    x U(0.9, 1.1) in flux.  Returns (image, background, inv_var, psf, sources, init)."""
    from .psf import CircularGaussianPSF
    rng = np.random.default_rng(seed)
    psf = CircularGaussianPSF(fwhm=2.5)
    src = simulate_sources(shape, n, rng=rng, flux=(1e2, 1e5), flux_distribution="loguniform")
    model = np.zeros(shape)
    render_sources(model, psf, src["y"], src["x"], src["flux"], model_radius=7)
    img = add_noise(model + 100.0, rng=rng, noise="poisson", gain=1.0)
    iv = 1.0 / (100.0 + model)
    init = dict(y=src["y"] + rng.normal(0, 0.3, n), x=src["x"] + rng.normal(0, 0.3, n),
                flux=src["flux"] * rng.uniform(0.9, 1.1, n))
    return img, np.full(shape, 100.0), iv, psf, src, init
