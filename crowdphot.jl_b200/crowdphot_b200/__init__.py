"""crowdphot_b200 -- B200 (sm_100a) drop-in for CrowdPhot.jl's PSF-fitting hot path.

Public API (names and keyword arguments follow the Julia package):
    fit_all_stars_simultaneous(image, psf, sources, fit_rad; ...) -> MultiPassPhotResult
    fit_star(model, image, inds; ...) -> (best_model, LMResult)
    fit_all_stars(image, psf, sources, fit_rad; n_passes, ...) -> MultiPassPhotResult
    fit_star_batch(model, cutouts; ...)  (many fit_star calls in one launch)
    fit_all_stars_simultaneous_batch(images, psf, sources_list, fit_rad; ...)
        (many small simultaneous fits in one launch, one thread block per group)
PSF types: CircularGaussianPSF, ImagePSF, GriddedPSFModel (of ImagePSF nodes),
CircularMoffatPSF (evaluation only, to tabulate empirical PSFs).
"""
from .psf import (AbstractPSFModel, ArgumentError, CircularGaussianPSF, CircularMoffatPSF, GriddedPSFModel,
                  ImagePSF, replace_params)
from .photometry import (BatchGraph, Context, CudaError, Request, Server, LMResult, MultiPassPhotResult, fit_all_stars_simultaneous,
                         fit_all_stars, fit_all_stars_simultaneous_batch, fit_groups_packed, fit_star, fit_star_batch,
                         fit_star_packed, get_context, lm_params, psf_descriptor, sim_params)
from ._abi import LIB_PATH, load_library
from .robust import FixedScale, HuberLoss, L2DistLoss, LogitDistLoss, MADScale, MScale, TukeyLoss

__all__ = [
    "AbstractPSFModel", "ArgumentError", "CircularGaussianPSF", "CircularMoffatPSF", "GriddedPSFModel", "ImagePSF",
    "replace_params", "BatchGraph", "Context", "Request", "Server", "CudaError", "LMResult", "MultiPassPhotResult", "fit_all_stars_simultaneous",
    "fit_all_stars", "fit_all_stars_simultaneous_batch", "fit_groups_packed",
    "fit_star", "fit_star_batch", "fit_star_packed", "get_context", "lm_params", "psf_descriptor", "sim_params", "LIB_PATH",
    "load_library", "L2DistLoss", "HuberLoss", "TukeyLoss", "LogitDistLoss", "MADScale", "FixedScale", "MScale",
]
