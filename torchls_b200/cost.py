"""Residual batches of the typed API: ``Cost`` and ``Cost.factory``.

The interface (field names, defaults, the decorator and the errors it raises)
is torchls ``cost.py:16-68``; a ``Cost`` is one batch of single-observation
residuals over ``Var`` handles (or ``("name", idx)`` bindings made by
``Problem.add_residual``) and data.
"""

from __future__ import annotations

from collections.abc import Callable
from dataclasses import dataclass
from functools import update_wrapper
from typing import Literal

from torch import Tensor

from .batching import AutoBatchSize, BatchSize
from .losses import Loss

JacMode = Literal["auto", "reverse", "forward"]
_JAC_MODES = frozenset(("auto", "reverse", "forward"))


def _positive_int(x) -> bool:
    return isinstance(x, int) and not isinstance(x, bool) and x > 0


@dataclass(frozen=True)
class Cost:
    """One batch of residuals; ``residual_fn`` sees one observation's values.

    ``args`` mixes variable handles and data. Data carries a leading
    observation axis (length one broadcasts) unless its ``in_dims`` entry is
    None (shared by all observations). ``jacobian_fn`` (optional) returns one
    raw-residual Jacobian per variable argument; ``loss`` then ``weights``
    shape each observation's contribution to the objective. ``batch_size``
    chunks the torch.func linearization of user residuals (None: one chunk).
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
        problems = []
        if not (self.loss is None or isinstance(self.loss, Loss)):
            raise TypeError("loss must be a Loss instance such as HuberLoss, or None")
        if self.jac_mode not in _JAC_MODES:
            problems.append("jac_mode must be auto, reverse or forward")
        if not (self.batch_size is None or isinstance(self.batch_size, AutoBatchSize)
                or _positive_int(self.batch_size)):
            problems.append("batch_size must be a positive integer, AutoBatchSize, or None")
        if self.in_dims is not None:
            ok = len(self.in_dims) == len(self.args) and all(d is None or d == 0 for d in self.in_dims)
            if not ok:
                problems.append("in_dims must contain one 0 or None per argument")
        if problems:
            raise ValueError(problems[0])

    @staticmethod
    def factory(fn=None, **options):
        """Turn a single-observation residual into a Cost builder:
        ``make = Cost.factory(residual, loss=...); make(var_a, var_b, data)``.
        Usable bare (``@Cost.factory``) or with options (``@Cost.factory(...)``)."""

        def builder_for(residual_fn):
            def build(*args):
                return Cost(residual_fn, args, **options)

            return update_wrapper(build, residual_fn)

        if fn is None:
            return builder_for
        return builder_for(fn)
