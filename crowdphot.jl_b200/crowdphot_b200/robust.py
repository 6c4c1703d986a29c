"""IRLS losses and scale estimators of CrowdPhot's lm_irls, as plain descriptors.

Mirrors the objects a Julia caller passes as ``reweight`` / ``scale_estimator``
(src/levenberg_marquardt.jl:105-355): ``L2DistLoss`` and ``HuberLoss(d)`` from
LossFunctions.jl, CrowdPhot's ``TukeyLoss(c)``, and ``MADScale()``,
``FixedScale(sigma)``, ``MScale(delta, tol, max_iter)``.  The arithmetic runs on
the device; these classes only carry the parameters across the C-ABI.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import _abi
from .psf import ArgumentError


@dataclass(frozen=True)
class L2DistLoss:
    """Squared loss: IRLS weight 1 (psi(r) = 2r, psi'(0) = 2)."""


@dataclass(frozen=True)
class HuberLoss:
    """Huber loss with crossover d: weight 1 for |r| <= d, d / |r| beyond."""
    d: float = 1.0


@dataclass(frozen=True)
class TukeyLoss:
    """Tukey's bisquare: weight (1 - (r/c)^2)^2 for |r| <= c, 0 beyond (c = 4.685)."""
    c: float = 4.685


@dataclass(frozen=True)
class LogitDistLoss:
    """LossFunctions.jl's logistic distance loss, -log(4 e^r / (1 + e^r)^2): weight
    tanh(r/2) / (r/2) (psi(r) = tanh(r/2), psi'(0) = 1/2)."""


@dataclass(frozen=True)
class MADScale:
    """1.4826 * median(|r - median(r)|)."""


@dataclass(frozen=True)
class FixedScale:
    sigma: float


@dataclass(frozen=True)
class MScale:
    """Huber's proposal-2 M-scale with the residual capped at 3 sigma."""
    delta: float = 0.5
    tol: float = 1.0e-6
    max_iter: int = 30


def set_irls(P, reweight, scale_estimator, weight_reset_tol):
    """Fill the IRLS fields of a cpb_lm_params (lm_irls's keyword checks, :431-449)."""
    wrt = float(weight_reset_tol)
    if not wrt >= 0:  # NaN fails this test first, as in the reference
        raise ArgumentError("`weight_reset_tol` must be non-negative")
    P.weight_reset_tol = wrt
    P.mscale_delta, P.mscale_tol, P.mscale_max_iter = 0.5, 1.0e-6, 30
    if reweight is None:
        P.reweight = _abi.CPB_LOSS_NONE
    elif isinstance(reweight, L2DistLoss):
        P.reweight = _abi.CPB_LOSS_L2DIST
    elif isinstance(reweight, HuberLoss):
        if not float(reweight.d) > 0:
            raise ArgumentError("Huber crossover parameter must be strictly positive.")
        P.reweight, P.loss_param = _abi.CPB_LOSS_HUBER, float(reweight.d)
    elif isinstance(reweight, TukeyLoss):
        P.reweight, P.loss_param = _abi.CPB_LOSS_TUKEY, float(reweight.c)
    elif isinstance(reweight, LogitDistLoss):
        P.reweight = _abi.CPB_LOSS_LOGITDIST
    else:
        raise ArgumentError(f"reweight loss {type(reweight).__name__} is not supported by the B200 path "
                            "(L2DistLoss, HuberLoss, TukeyLoss and LogitDistLoss are)")
    if scale_estimator is None:
        P.scale_estimator = _abi.CPB_SCALE_AUTO
    elif isinstance(scale_estimator, MADScale):
        P.scale_estimator = _abi.CPB_SCALE_MAD
    elif isinstance(scale_estimator, FixedScale):
        P.scale_estimator, P.scale_value = _abi.CPB_SCALE_FIXED, float(scale_estimator.sigma)
    elif isinstance(scale_estimator, MScale):
        P.scale_estimator = _abi.CPB_SCALE_MSCALE
        P.mscale_delta, P.mscale_tol = float(scale_estimator.delta), float(scale_estimator.tol)
        P.mscale_max_iter = int(scale_estimator.max_iter)
    else:
        raise ArgumentError(f"scale estimator {type(scale_estimator).__name__} is not supported by the B200 path")
    return P


__all__ = ["L2DistLoss", "HuberLoss", "TukeyLoss", "LogitDistLoss", "MADScale", "FixedScale", "MScale", "set_irls"]
