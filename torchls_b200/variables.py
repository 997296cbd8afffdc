"""Variable types, value containers and the tangent layout.

Interface follows torchls ``variables.py``: ``Var`` subclasses are declared
with ``default_factory``, ``tangent_dim``, ``retract_fn`` and an optional
``retract_jvp_fn`` (torchls variables.py:18-55); ``VarValues.make`` stacks
values by type sorted by ID (variables.py:189-216); ``VariableLayout`` places
each group at ``offset`` with ``count * dim`` tangent entries
(variables.py:100-117).
"""

from __future__ import annotations

import math
from collections.abc import Callable, Iterable, Mapping
from dataclasses import dataclass

import torch
from torch import Tensor


def as_ids(ids) -> Tensor:
    """Validate scalar or 1-D integer IDs and return them as int64."""
    out = torch.as_tensor(ids)
    if out.dtype not in (torch.int32, torch.int64) or out.ndim > 1:
        raise ValueError("Variable IDs must be scalar or 1D integer tensors")
    return out.to(dtype=torch.long)


@dataclass(frozen=True)
class Var:
    """Symbolic variable(s) identified by subclass and integer ID(s)."""

    id: int | Tensor

    def __init_subclass__(
        cls,
        *,
        default_factory: Callable[[], Tensor],
        tangent_dim: int | None = None,
        retract_fn: Callable[[Tensor, Tensor], Tensor] | None = None,
        retract_jvp_fn: Callable[[Tensor, Tensor], Tensor] | None = None,
        **kwargs,
    ):
        super().__init_subclass__(**kwargs)
        proto = default_factory()
        if not isinstance(proto, Tensor) or not proto.is_floating_point():
            raise TypeError("default_factory must return a floating point Tensor")
        if (tangent_dim is None) != (retract_fn is None):
            raise ValueError("Specify tangent_dim and retract_fn together")
        if retract_jvp_fn is not None and retract_fn is None:
            raise ValueError("retract_jvp_fn requires a manifold retract_fn")
        if retract_jvp_fn is not None and not callable(retract_jvp_fn):
            raise TypeError("retract_jvp_fn must be callable")
        cls.default_factory = staticmethod(default_factory)
        cls.is_euclidean = retract_fn is None
        cls.tangent_dim = proto.numel() if tangent_dim is None else tangent_dim
        if cls.tangent_dim <= 0:
            raise ValueError("tangent_dim must be positive")
        if retract_fn is None:
            cls.retract_fn = staticmethod(lambda x, d: x + d.reshape(x.shape))
        else:
            cls.retract_fn = staticmethod(retract_fn)
        # Never inherited: a new retraction needs its own derivative.
        cls.retract_jvp_fn = staticmethod(retract_jvp_fn) if retract_jvp_fn is not None else None
        # CUDA retraction kind; Euclidean groups use "euclidean", custom
        # manifolds are retracted with their torch retract_fn.
        cls.cuda_kind = "euclidean" if retract_fn is None else None

    def __post_init__(self):
        as_ids(self.id)

    def __getitem__(self, index) -> Var:
        return type(self)(as_ids(self.id)[index])

    def with_value(self, value: Tensor) -> VarWithValue:
        return VarWithValue(self, value)


@dataclass(frozen=True)
class VarWithValue:
    variable: Var
    value: Tensor


@dataclass(frozen=True)
class ParameterRef:
    """A ``("name", index)`` binding made by :meth:`Problem.add_residual`."""

    name: str
    id: int | Tensor

    def __post_init__(self):
        as_ids(self.id)


@dataclass(frozen=True)
class EuclideanGroup:
    """Parameterisation of a named group without a declared manifold."""

    shape: tuple[int, ...]
    is_euclidean = True
    retract_jvp_fn = None
    cuda_kind = "euclidean"

    @property
    def tangent_dim(self) -> int:
        return math.prod(self.shape)

    def default_factory(self) -> Tensor:
        return torch.zeros(self.shape)

    @staticmethod
    def retract_fn(value, delta):
        return value + delta.reshape(value.shape)


@dataclass(frozen=True)
class VariableLayout:
    """One variable group's place in the global tangent vector."""

    var_type: object
    ids: Tensor
    offset: int
    name: str | None = None

    @property
    def key(self):
        return self.var_type if self.name is None else self.name

    @property
    def count(self) -> int:
        return self.ids.numel()

    @property
    def dim(self) -> int:
        return self.var_type.tangent_dim

    @property
    def size(self) -> int:
        return self.count * self.dim


def _retract_group(entry: VariableLayout, value: Tensor, delta: Tensor) -> Tensor:
    from .kernels import retract_group

    return retract_group(entry, value, delta.reshape(entry.count, entry.dim))


class NamedValues:
    """Solver state keyed by parameter-group name (the ``Problem`` API)."""

    def __init__(self, values: Mapping[str, Tensor], layout: tuple[VariableLayout, ...]):
        if not layout or set(values) != {e.key for e in layout}:
            raise ValueError("Parameter names do not match the analyzed problem")
        first = values[layout[0].key]
        for e in layout:
            v = values[e.key]
            expected = (e.count, *e.var_type.default_factory().shape)
            if not isinstance(v, Tensor) or tuple(v.shape) != expected:
                raise ValueError(f"{e.key}: expected parameter tensor of shape {expected}")
            if v.dtype not in (torch.float32, torch.float64):
                raise ValueError("Use float32 or float64 for least squares")
            if v.dtype != first.dtype or v.device != first.device:
                raise ValueError("All parameters must have the same dtype and device")
        self._values = dict(values)
        self._ids = {e.key: e.ids for e in layout}
        self._layout = layout

    @property
    def dtype(self):
        return next(iter(self._values.values())).dtype

    @property
    def device(self):
        return next(iter(self._values.values())).device

    def detach(self):
        return NamedValues({k: v.detach() for k, v in self._values.items()}, self._layout)

    def retract(self, tangent: Tensor, layout) -> NamedValues:
        out = {}
        for e in layout:
            delta = tangent[e.offset : e.offset + e.size]
            out[e.key] = _retract_group(e, self._values[e.key], delta)
        return NamedValues(out, layout)


class VarValues:
    """Values stacked per variable type and sorted by ID (the typed API)."""

    def __init__(self, values: dict, ids: dict):
        if not values or values.keys() != ids.keys():
            raise ValueError("Values and IDs must contain the same nonempty types")
        self._values = dict(values)
        self._ids = {k: as_ids(v).reshape(-1).cpu() for k, v in ids.items()}
        first = next(iter(values.values()))
        for key, value in values.items():
            expected = (len(self._ids[key]), *key.default_factory().shape)
            if tuple(value.shape) != expected:
                raise ValueError(f"{key.__name__}: expected values of shape {expected}")
            if (
                not value.is_floating_point()
                or value.dtype != first.dtype
                or value.device != first.device
            ):
                raise ValueError("All variable values must have the same floating dtype and device")
            if value.dtype not in (torch.float32, torch.float64):
                raise ValueError("Use float32 or float64 for least squares")
            ids_k = self._ids[key]
            if len(ids_k) == 0 or not bool(torch.all(ids_k[1:] > ids_k[:-1])):
                raise ValueError("Variable IDs must be nonempty, sorted and unique")

    @classmethod
    def make(cls, variables: Iterable[Var | VarWithValue]) -> VarValues:
        vals: dict = {}
        idss: dict = {}
        for item in variables:
            var = item.variable if isinstance(item, VarWithValue) else item
            key = type(var)
            ids = as_ids(var.id)
            shape = key.default_factory().shape
            if isinstance(item, VarWithValue):
                value = item.value
                if tuple(value.shape) != (*ids.shape, *shape):
                    raise ValueError(
                        f"{key.__name__}: expected shape {(*ids.shape, *shape)}, got {tuple(value.shape)}"
                    )
            else:
                value = key.default_factory().to(device=ids.device).expand((*ids.shape, *shape))
            flat = ids.reshape(-1)
            vals.setdefault(key, []).append(value.reshape(flat.numel(), *shape))
            idss.setdefault(key, []).append(flat.cpu())
        out_v, out_i = {}, {}
        for key, parts in vals.items():
            ids = torch.cat(idss[key])
            order = ids.argsort()
            out_i[key] = ids[order]
            stacked = torch.cat(parts)
            out_v[key] = stacked[order.to(stacked.device)]
        return cls(out_v, out_i)

    @property
    def dtype(self):
        return next(iter(self._values.values())).dtype

    @property
    def device(self):
        return next(iter(self._values.values())).device

    def __getitem__(self, var):
        if isinstance(var, type):
            return self._values[var]
        ids = as_ids(var.id).cpu()
        known = self._ids[type(var)]
        pos = torch.searchsorted(known, ids)
        if bool(torch.any(pos >= len(known))) or not torch.equal(known[pos.clamp_max(len(known) - 1)], ids):
            raise KeyError(f"Unknown {type(var).__name__} ID")
        return self._values[type(var)][pos.to(self.device)]

    def to(self, *args, **kwargs) -> VarValues:
        return VarValues({k: x.to(*args, **kwargs) for k, x in self._values.items()}, self._ids)

    def detach(self) -> VarValues:
        return VarValues({k: x.detach() for k, x in self._values.items()}, self._ids)

    def retract(self, tangent: Tensor, layout) -> VarValues:
        out = {}
        for e in layout:
            delta = tangent[e.offset : e.offset + e.size]
            out[e.var_type] = _retract_group(e, self._values[e.var_type], delta)
        return VarValues(out, self._ids)
