"""Robust losses on each observation's squared residual norm s = |r|^2.

Interface of torchls ``losses.py``: F = 0.5 * sum rho(s); ``evaluate`` returns
(rho, rho', rho''). ``HuberLoss`` is evaluated inside the CUDA linearization
and trial kernels; any other ``Loss`` subclass is evaluated by its own torch
``evaluate`` on the device and its (rho', rho'') feed the kernel's clamped
curvature correction (torchls losses.py:30-50).
"""

from __future__ import annotations

import math
from abc import ABC, abstractmethod
from dataclasses import dataclass

import torch
from torch import Tensor


class Loss(ABC):
    """Define rho(s), rho'(s), rho''(s) for F = 0.5 * sum(rho(|r_i|^2)).

    Losses must have nonnegative values and first derivatives. Linearization
    uses the clamped curvature correction: nonpositive rho'' is ignored;
    positive rho'' receives the full rank-one correction.
    """

    cuda_kind = "generic"

    @abstractmethod
    def evaluate(self, squared_norm: Tensor) -> tuple[Tensor, Tensor, Tensor]:
        """Return the loss value and first two derivatives with respect to s."""

    def value(self, squared_norm: Tensor) -> Tensor:
        return self.evaluate(squared_norm)[0]


@dataclass(frozen=True)
class HuberLoss(Loss):
    """Huber loss on the norm of a complete residual block.

    rho(s) = s for |r| <= delta, otherwise 2 * delta * |r| - delta^2
    (torchls losses.py:56-107). The robust model scales residuals and
    Jacobians by sqrt(rho'(s)); trial steps use a divided-difference reduction.
    """

    delta: float = 1.0
    cuda_kind = "huber"

    def __post_init__(self):
        if not math.isfinite(self.delta) or self.delta <= 0:
            raise ValueError("Huber delta must be finite and positive")

    def evaluate(self, squared_norm: Tensor) -> tuple[Tensor, Tensor, Tensor]:
        safe = squared_norm.clamp_min(torch.finfo(squared_norm.dtype).tiny)
        norm = safe.sqrt()
        outlier = squared_norm > self.delta * self.delta
        first = torch.where(outlier, self.delta / norm, torch.ones_like(norm))
        value = torch.where(outlier, self.delta * (2 * norm - self.delta), squared_norm)
        second = torch.where(outlier, -0.5 * first / safe, torch.zeros_like(norm))
        return value, first, second

    def value(self, squared_norm: Tensor) -> Tensor:
        norm = squared_norm.clamp_min(torch.finfo(squared_norm.dtype).tiny).sqrt()
        return torch.where(squared_norm > self.delta * self.delta, self.delta * (2 * norm - self.delta),
                           squared_norm)
