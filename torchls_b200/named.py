"""Name-and-index modelling API (interface of torchls ``named.py:24-154``)."""

from __future__ import annotations

from collections.abc import Callable, Mapping

import torch
from torch import Tensor

from .batching import BatchSize
from .cost import Cost, JacMode
from .losses import Loss
from .problem import AnalyzedLeastSquaresProblem
from .variables import EuclideanGroup, NamedValues, ParameterRef, Var, VariableLayout, as_ids


class Problem:
    """Own parameter tensors by name and bind residual inputs with (name, index).

    Each parameter tensor has shape [count, *storage]. Unspecified groups are
    Euclidean; ``manifolds`` assigns Var parameterisations, e.g.
    {"cams": SE3Var}. ``solve`` returns a dict and writes the solved tensors
    back into ``parameters`` (so a second solve warm-starts).
    """

    def __init__(self, parameters: Mapping[str, Tensor], *, manifolds: Mapping[str, type[Var]] | None = None):
        self.parameters = dict(parameters)
        self.manifolds = dict(manifolds or {})
        self._costs: list[Cost] = []
        self._analyzed = None
        self._signature = None
        self.last_summary = None

    def add_residual(self, residual_fn: Callable[..., Tensor], *args, jac_mode: JacMode = "auto",
                     batch_size: BatchSize = None, in_dims: tuple[int | None, ...] | None = None,
                     jacobian_fn: Callable[..., tuple[Tensor, ...]] | None = None, loss: Loss | None = None,
                     weights: Tensor | float | None = None) -> Problem:
        """Add a batch of residuals; ("name", indices) selects optimisable rows.

        Other arguments are constant data. Indices are copied when the batch is
        added. ``loss`` applies to each observation's residual block; weights
        scale the loss (scalar or one per observation).
        """
        if not callable(residual_fn):
            raise TypeError("The first argument must be a residual function")
        bound = tuple(
            ParameterRef(a[0], as_ids(a[1]).detach().cpu().clone())
            if isinstance(a, tuple) and len(a) == 2 and isinstance(a[0], str) else a
            for a in args
        )
        self._costs.append(Cost(residual_fn, bound, jac_mode, batch_size, in_dims, jacobian_fn, loss, weights))
        self._analyzed = None
        return self

    def _ensure_analyzed(self):
        if not self.parameters or not self._costs:
            raise ValueError("A problem needs parameters and residuals")
        if set(self.manifolds) - set(self.parameters):
            raise ValueError("Manifold names must refer to declared parameter groups")
        signature, specs = [], []
        for name, value in self.parameters.items():
            if not isinstance(name, str) or not name:
                raise ValueError("Parameter group names must be nonempty strings")
            if not isinstance(value, Tensor) or value.ndim < 1 or value.numel() == 0:
                raise ValueError(f"{name}: expected a nonempty tensor with a leading parameter axis")
            spec = self.manifolds.get(name)
            if spec is None:
                spec = EuclideanGroup(tuple(value.shape[1:]))
            elif not isinstance(spec, type) or not issubclass(spec, Var):
                raise TypeError(f"{name}: manifold must be a Var parameterization such as SE3Var")
            specs.append(spec)
            signature.append((name, tuple(value.shape), spec))
        signature = tuple(signature)
        if self._analyzed is None or signature != self._signature:
            layout, offset = [], 0
            for (name, value), spec in zip(self.parameters.items(), specs, strict=True):
                entry = VariableLayout(spec, torch.arange(value.shape[0]), offset, name=name)
                layout.append(entry)
                offset += entry.count * entry.dim
            layout = tuple(layout)
            NamedValues(self.parameters, layout)
            self._analyzed = AnalyzedLeastSquaresProblem(layout, tuple(self._costs), offset)
            self._signature = signature
        return self._analyzed

    def refresh_data(self) -> Problem:
        """Re-read residual data and weights after in-place changes, keeping the
        analysis (structure, Schur plans) of the unchanged sparsity pattern."""
        if self._analyzed is not None:
            self._analyzed.refresh_data()
        return self

    def analyze(self) -> Problem:
        self._state(None)
        return self

    @property
    def tangent_dim(self):
        return self._ensure_analyzed().tangent_dim

    def _state(self, parameters):
        analyzed = self._ensure_analyzed()
        return analyzed, NamedValues(self.parameters if parameters is None else parameters, analyzed.layout)

    def residuals(self, parameters: Mapping[str, Tensor] | None = None):
        analyzed, state = self._state(parameters)
        return analyzed.residuals(state)

    def cost(self, parameters: Mapping[str, Tensor] | None = None):
        analyzed, state = self._state(parameters)
        return analyzed.cost(state)

    def linearize(self, parameters: Mapping[str, Tensor] | None = None, **kwargs):
        analyzed, state = self._state(parameters)
        return analyzed.linearize(state, **kwargs)

    def solve(self, *, return_summary: bool = False, **options):
        analyzed, initial = self._state(None)
        solution, summary = analyzed.solve(initial, return_summary=True, **options)
        result = dict(solution._values)
        self.parameters.update(result)
        self.last_summary = summary
        return (result, summary) if return_summary else result
