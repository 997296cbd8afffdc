"""Box bounds on Euclidean groups (interface of torchls ``bounds.py:10-75``).

The active set masks gradient and Jacobian columns; the projected retraction
runs in the CUDA retraction kernel (clamp + effective step).
"""

from __future__ import annotations

from collections.abc import Mapping

import torch

from . import _lib as L
from .variables import NamedValues, VarValues


class BoundsPlan:
    def __init__(self, bounds, layout, initial):
        if not isinstance(bounds, Mapping):
            raise TypeError("bounds must map parameter names or Var types to (lower, upper)")
        entries = {e.key: e for e in layout}
        self.groups = []
        self.layout = layout
        for key, pair in bounds.items():
            if key not in entries:
                raise ValueError(f"Bounds refer to undeclared parameter group {key!r}")
            entry = entries[key]
            if not getattr(entry.var_type, "is_euclidean", False):
                raise ValueError("Bounds require Euclidean groups without a custom retraction")
            if not isinstance(pair, (tuple, list)) or len(pair) != 2:
                raise ValueError("Each bounds entry must be a (lower, upper) pair")
            value = initial._values[key]
            limits = []
            for limit, default in zip(pair, (-torch.inf, torch.inf), strict=True):
                t = torch.as_tensor(default if limit is None else limit, dtype=torch.float64, device=value.device)
                try:
                    limits.append(torch.broadcast_to(t, value.shape).contiguous().clone())
                except RuntimeError as err:
                    raise ValueError(f"Bounds for {key!r} do not broadcast to {tuple(value.shape)}") from err
            lo, hi = limits
            if bool(torch.isnan(lo).any() | torch.isnan(hi).any() | (lo > hi).any()):
                raise ValueError("Bounds must be ordered and cannot contain NaN")
            v = value.double()
            if bool(((v < lo) | (v > hi)).any()):
                raise ValueError(f"Initial values of {key!r} are outside their bounds")
            self.groups.append((entry, lo, hi))

    def free_mask(self, values, gradient):
        """1 for free columns, 0 for active ones (bounds.py:44-56), float64."""
        mask = torch.ones_like(gradient, dtype=torch.float64)
        for e, lo, hi in self.groups:
            a, b = e.offset, e.offset + e.size
            v = values._values[e.key].double()
            g = gradient[a:b].reshape(v.shape)
            active = (lo == hi) | ((v <= lo) & (g > 0)) | ((v >= hi) & (g < 0))
            mask[a:b] = (~active).reshape(-1).to(torch.float64)
        return mask

    def projected_gradient(self, values, gradient):
        return gradient * self.free_mask(values, gradient)

    def retract(self, values, tangent):
        """Retract, clamp bounded groups and return the effective step (bounds.py:61-75)."""
        from .kernels import retract_group

        bounded = {e.key: (lo, hi) for e, lo, hi in self.groups}
        effective = tangent.to(torch.float64).clone()
        out = {}
        for e in self.layout:
            v = values._values[e.key]
            d = effective[e.offset : e.offset + e.size]
            if e.key in bounded:
                lo, hi = bounded[e.key]
                step = torch.empty_like(d)
                out[e.key] = retract_group(e, v, d.view(e.count, e.dim), lo, hi, step)
                effective[e.offset : e.offset + e.size] = step
            else:
                out[e.key] = retract_group(e, v, d.view(e.count, e.dim))
        if isinstance(values, VarValues):
            return VarValues(out, values._ids), effective
        return NamedValues(out, self.layout), effective
