"""``Cost`` records and the ``Cost.factory`` decorator (torchls cost.py:16-68)."""

from __future__ import annotations

from collections.abc import Callable
from dataclasses import dataclass
from functools import wraps
from typing import Literal

from torch import Tensor

from .batching import AutoBatchSize, BatchSize
from .losses import Loss

JacMode = Literal["auto", "reverse", "forward"]


@dataclass(frozen=True)
class Cost:
    """One batch of residuals; functions receive local values, not Var handles.

    Tensor data defaults to a leading observation axis (length one broadcasts);
    ``in_dims=None`` marks data shared by every observation. Weights scale each
    observation's objective after its loss.
    """

    residual_fn: Callable[..., Tensor]
    args: tuple
    jac_mode: JacMode = "auto"
    batch_size: BatchSize = None
    in_dims: tuple[int | None, ...] | None = None
    jacobian_fn: Callable[..., tuple[Tensor, ...]] | None = None
    loss: Loss | None = None
    weights: Tensor | float | None = None

    def __post_init__(self):
        if self.loss is not None and not isinstance(self.loss, Loss):
            raise TypeError("loss must be a Loss instance such as HuberLoss, or None")
        if self.jac_mode not in ("auto", "reverse", "forward"):
            raise ValueError("jac_mode must be auto, reverse or forward")
        if self.batch_size is not None and not isinstance(self.batch_size, AutoBatchSize):
            if isinstance(self.batch_size, bool) or not isinstance(self.batch_size, int) or self.batch_size <= 0:
                raise ValueError("batch_size must be a positive integer, AutoBatchSize, or None")
        if self.in_dims is not None and (
            len(self.in_dims) != len(self.args) or any(x not in (0, None) for x in self.in_dims)
        ):
            raise ValueError("in_dims must contain one 0 or None per argument")

    @staticmethod
    def factory(fn=None, **options):
        """Decorate a single-observation residual to create batched Costs."""

        def decorate(residual_fn):
            @wraps(residual_fn)
            def make(*args):
                return Cost(residual_fn, args, **options)

            return make

        return decorate(fn) if fn is not None else decorate
