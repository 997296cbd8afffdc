"""Name-and-index modelling API (the interface of torchls ``named.py:24-154``).

A ``Problem`` owns parameter tensors by group name; residual batches bind
rows of a group with ``("name", indices)``. The analysis (tangent layout,
index maps, device structures, Schur plans) is built on first use and reused
while the groups keep their names, shapes and parameterizations; adding a
residual batch discards it.
"""

from __future__ import annotations

from collections.abc import Callable, Mapping

import torch
from torch import Tensor

from .batching import BatchSize
from .cost import Cost, JacMode
from .losses import Loss
from .problem import AnalyzedLeastSquaresProblem
from .variables import NamedValues, ParameterRef, Var, VariableLayout, as_ids, euclidean_type


def _binding(arg):
    """``("name", indices)`` becomes a ParameterRef with a private int64 copy of
    the indices (later edits of the caller's tensor do not change the problem);
    any other argument is data and passes through."""
    if isinstance(arg, tuple) and len(arg) == 2 and isinstance(arg[0], str):
        return ParameterRef(arg[0], as_ids(arg[1]).detach().cpu().clone())
    return arg


class Problem:
    """Parameter tensors by name, residual batches bound by (name, indices).

    Each tensor has shape [count, *storage]. A group without an entry in
    ``manifolds`` is a vector space; ``manifolds={"cams": SE3Var}`` gives it a
    Var parameterization. ``solve`` returns a dict of solved tensors and also
    stores them in ``parameters`` (a second solve warm-starts from them).
    """

    def __init__(self, parameters: Mapping[str, Tensor], *, manifolds: Mapping[str, type[Var]] | None = None):
        self.parameters = dict(parameters)
        self.manifolds = dict(manifolds or {})
        self.last_summary = None
        self._costs: list[Cost] = []
        self._cache: tuple | None = None  # (signature, analysed problem)

    def add_residual(self, residual_fn: Callable[..., Tensor], *args, jac_mode: JacMode = "auto",
                     batch_size: BatchSize = None, in_dims: tuple[int | None, ...] | None = None,
                     jacobian_fn: Callable[..., tuple[Tensor, ...]] | None = None, loss: Loss | None = None,
                     weights: Tensor | float | None = None) -> Problem:
        """Append one residual batch and return the problem (chainable).

        ``residual_fn`` takes one observation's arguments; ``("name", idx)``
        arguments are optimised rows, everything else is data with a leading
        observation axis (or shared, ``in_dims`` None). ``loss`` acts on each
        observation's whole residual; ``weights`` (scalar or per observation)
        scale the loss.
        """
        if not callable(residual_fn):
            raise TypeError("The first argument must be a residual function")
        self._costs.append(Cost(residual_fn, tuple(map(_binding, args)), jac_mode=jac_mode, batch_size=batch_size,
                                in_dims=in_dims, jacobian_fn=jacobian_fn, loss=loss, weights=weights))
        self._cache = None
        return self

    # ------------------------------------------------------------------ analysis
    def _signature(self) -> tuple:
        """(name, shape, parameterization) per group, validated."""
        if not (self.parameters and self._costs):
            raise ValueError("A problem needs parameters and residuals")
        unknown = set(self.manifolds).difference(self.parameters)
        if unknown:
            raise ValueError("Manifold names must refer to declared parameter groups")
        out = []
        for name, value in self.parameters.items():
            if not (isinstance(name, str) and name):
                raise ValueError("Parameter group names must be nonempty strings")
            if not (isinstance(value, Tensor) and value.ndim >= 1 and value.numel() > 0):
                raise ValueError(f"{name}: expected a nonempty tensor with a leading parameter axis")
            kind = self.manifolds.get(name)
            if kind is None:
                kind = euclidean_type(tuple(value.shape[1:]))
            elif not (isinstance(kind, type) and issubclass(kind, Var)):
                raise TypeError(f"{name}: manifold must be a Var parameterization such as SE3Var")
            out.append((name, tuple(value.shape), kind))
        return tuple(out)

    def _ensure_analyzed(self) -> AnalyzedLeastSquaresProblem:
        sig = self._signature()
        if self._cache is None or self._cache[0] != sig:
            offsets = [0]
            for _, shape, kind in sig:
                offsets.append(offsets[-1] + shape[0] * kind.tangent_dim)
            layout = tuple(VariableLayout(kind, torch.arange(shape[0]), off, name=name)
                           for (name, shape, kind), off in zip(sig, offsets))
            NamedValues(self.parameters, layout)  # dtype / device / shape checks
            self._cache = (sig, AnalyzedLeastSquaresProblem(layout, tuple(self._costs), offsets[-1]))
        return self._cache[1]

    def analyze(self) -> Problem:
        """Build the analysis now (it is otherwise built on first use)."""
        self._ensure_analyzed()
        return self

    def refresh_data(self) -> Problem:
        """Re-read residual data and weights after in-place edits, keeping the
        analysis of the unchanged sparsity pattern."""
        if self._cache is not None:
            self._cache[1].refresh_data()
        return self

    @property
    def tangent_dim(self) -> int:
        return self._ensure_analyzed().tangent_dim

    def _state(self, parameters):
        analyzed = self._ensure_analyzed()
        return analyzed, NamedValues(self.parameters if parameters is None else parameters, analyzed.layout)

    # ------------------------------------------------------------------ evaluation
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
        analyzed, start = self._state(None)
        solution, summary = analyzed.solve(start, return_summary=True, **options)
        solved = dict(solution._values)
        self.parameters.update(solved)
        self.last_summary = summary
        if return_summary:
            return solved, summary
        return solved
