"""Variable types, value containers and the tangent layout.

The public surface is the one torchls users program against: ``Var``
subclasses declared with class keywords (``default_factory``,
``tangent_dim``, ``retract_fn``, ``retract_jvp_fn``; torchls
variables.py:18-55), ``VarValues.make`` (values stacked per type, sorted by
ID; variables.py:189-216) and ``VariableLayout`` (group g occupies
``[offset, offset + count * dim)`` of the tangent vector; variables.py:100-117).
The layout rule and the ID order are formats that results depend on, so they
are kept; everything else here is this package's own structure:

* every variable type carries one ``Parameterization`` record, and the class
  attributes other modules read (``default_factory``, ``tangent_dim``,
  ``retract_fn``, ``retract_jvp_fn``, ``is_euclidean``, ``cuda_kind``) are
  views of it;
* a named parameter group without a declared manifold gets a real ``Var``
  subclass from ``euclidean_type(shape)`` (one class per storage shape);
* ``NamedValues`` (keyed by group name) and ``VarValues`` (keyed by type)
  share one base class that validates, detaches and retracts.
"""

from __future__ import annotations

import functools
from collections import defaultdict
from collections.abc import Callable, Iterable, Mapping
from dataclasses import dataclass
from typing import NamedTuple

import torch
from torch import Tensor

_INDEX_DTYPES = (torch.int32, torch.int64)
_VALUE_DTYPES = (torch.float32, torch.float64)


def as_ids(ids) -> Tensor:
    """Scalar or 1-D integer IDs as int64; anything else raises ValueError."""
    t = torch.as_tensor(ids)
    if t.ndim <= 1 and t.dtype in _INDEX_DTYPES:
        return t.long()
    raise ValueError("Variable IDs must be scalar or 1D integer tensors")


# ---------------------------------------------------------------- parameterizations
@dataclass(frozen=True)
class Parameterization:
    """Storage and update rule of one variable type.

    ``retract`` is None for a vector space (update by addition);
    ``retract_jvp`` is the first-order chart D_delta retract(x, delta) at 0,
    used by linearization when present.
    """

    make_default: Callable[[], Tensor]
    storage_shape: tuple[int, ...]
    tangent_dim: int
    retract: Callable[[Tensor, Tensor], Tensor] | None
    retract_jvp: Callable[[Tensor, Tensor], Tensor] | None

    @staticmethod
    def declare(default_factory, tangent_dim, retract_fn, retract_jvp_fn) -> Parameterization:
        sample = default_factory()
        if not (isinstance(sample, Tensor) and sample.is_floating_point()):
            raise TypeError("default_factory must return a floating point Tensor")
        if (tangent_dim is None) is not (retract_fn is None):
            raise ValueError("Specify tangent_dim and retract_fn together")
        if retract_jvp_fn is not None:
            if retract_fn is None:
                raise ValueError("retract_jvp_fn requires a manifold retract_fn")
            if not callable(retract_jvp_fn):
                raise TypeError("retract_jvp_fn must be callable")
        dim = sample.numel() if tangent_dim is None else int(tangent_dim)
        if dim <= 0:
            raise ValueError("tangent_dim must be positive")
        return Parameterization(default_factory, tuple(sample.shape), dim, retract_fn, retract_jvp_fn)

    def retract_value(self, value: Tensor, delta: Tensor) -> Tensor:
        if self.retract is None:
            return value + delta.reshape(value.shape)
        return self.retract(value, delta)


class Var:
    """Symbolic variable(s): a subclass (the type) and integer ID(s).

    Subclasses declare their parameterization with class keywords, e.g.
    ``class SE3Var(Var, default_factory=..., tangent_dim=6, retract_fn=...)``.
    The retraction derivative is never inherited: a subclass that changes the
    retraction must give its own ``retract_jvp_fn``.
    """

    __slots__ = ("id",)

    def __init_subclass__(cls, *, default_factory, tangent_dim=None, retract_fn=None, retract_jvp_fn=None,
                          **kwargs):
        super().__init_subclass__(**kwargs)
        param = Parameterization.declare(default_factory, tangent_dim, retract_fn, retract_jvp_fn)
        cls.parameterization = param
        cls.default_factory = staticmethod(param.make_default)
        cls.tangent_dim = param.tangent_dim
        cls.is_euclidean = param.retract is None
        cls.retract_fn = staticmethod(param.retract_value)
        cls.retract_jvp_fn = None if param.retract_jvp is None else staticmethod(param.retract_jvp)
        # kind of the CUDA retraction; known groups set their own tag, other
        # manifolds are retracted with their torch retract_fn
        cls.cuda_kind = "euclidean" if param.retract is None else None

    def __init__(self, id):
        as_ids(id)
        object.__setattr__(self, "id", id)

    def __setattr__(self, name, value):
        raise AttributeError("Var handles are immutable")

    def __eq__(self, other):
        return type(other) is type(self) and torch.equal(as_ids(self.id), as_ids(other.id))

    def __hash__(self):
        return hash((type(self), tuple(as_ids(self.id).reshape(-1).tolist())))

    def __repr__(self):
        return f"{type(self).__name__}({self.id!r})"

    def __getitem__(self, index) -> Var:
        return type(self)(as_ids(self.id)[index])

    def with_value(self, value: Tensor) -> VarWithValue:
        return VarWithValue(self, value)


class VarWithValue(NamedTuple):
    """A variable handle paired with its initial value(s)."""

    variable: Var
    value: Tensor


class ParameterRef(NamedTuple):
    """A ``("name", indices)`` binding made by ``Problem.add_residual``; the
    indices are validated int64 (``as_ids``) when the binding is made."""

    name: str
    id: Tensor


@functools.lru_cache(maxsize=None)
def euclidean_type(shape: tuple[int, ...]) -> type[Var]:
    """The vector-space ``Var`` type of a named group whose rows have storage
    ``shape`` (one class per shape, so analyses of equal shapes compare equal)."""
    shape = tuple(int(s) for s in shape)
    return type(f"Euclidean{'x'.join(map(str, shape)) or 'Scalar'}", (Var,), {"__slots__": ()},
                default_factory=lambda: torch.zeros(shape))


# ---------------------------------------------------------------- tangent layout
class VariableLayout(NamedTuple):
    """One variable group's place in the global tangent vector."""

    var_type: type
    ids: Tensor
    offset: int
    name: str | None = None

    @property
    def key(self):
        """The group's key in a values container: its name, else its type."""
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


# ---------------------------------------------------------------- value containers
class _ValueSet:
    """Stacked values per group key with their IDs; all groups share one
    floating dtype (float32 or float64) and one device."""

    def __init__(self, values: Mapping, ids: Mapping, expected_rows: Callable, label: Callable):
        self._values = dict(values)
        self._ids = dict(ids)
        ref = None
        for key, value in self._values.items():
            rows = expected_rows(key)
            if not isinstance(value, Tensor) or tuple(value.shape) != rows:
                raise ValueError(f"{label(key)}: expected values of shape {rows}")
            if value.dtype not in _VALUE_DTYPES:
                raise ValueError("Use float32 or float64 for least squares")
            ref = ref if ref is not None else value
            if (value.dtype, value.device) != (ref.dtype, ref.device):
                raise ValueError("All values must share one floating dtype and one device")

    @property
    def dtype(self):
        return next(iter(self._values.values())).dtype

    @property
    def device(self):
        return next(iter(self._values.values())).device

    def _retracted(self, tangent: Tensor, layout) -> dict:
        return {e.key: _retract_group(e, self._values[e.key], tangent[e.offset : e.offset + e.size])
                for e in layout}


class NamedValues(_ValueSet):
    """Solver state keyed by parameter-group name (the ``Problem`` API)."""

    def __init__(self, values: Mapping[str, Tensor], layout: tuple[VariableLayout, ...]):
        by_key = {e.key: e for e in layout}
        if not layout or set(values) != set(by_key):
            raise ValueError("Parameter names do not match the analyzed problem")
        super().__init__(values, {k: e.ids for k, e in by_key.items()},
                         lambda k: (by_key[k].count, *by_key[k].var_type.default_factory().shape), str)
        self._layout = layout

    def detach(self) -> NamedValues:
        return NamedValues({k: v.detach() for k, v in self._values.items()}, self._layout)

    def retract(self, tangent: Tensor, layout) -> NamedValues:
        return NamedValues(self._retracted(tangent, layout), layout)


class VarValues(_ValueSet):
    """Values stacked per variable type, rows sorted by ID (the typed API)."""

    def __init__(self, values: dict, ids: dict):
        if not values or set(values) != set(ids):
            raise ValueError("Values and IDs must contain the same nonempty types")
        ids = {t: as_ids(i).reshape(-1).cpu() for t, i in ids.items()}
        for t, i in ids.items():
            if i.numel() == 0 or bool((i[1:] <= i[:-1]).any()):
                raise ValueError("Variable IDs must be nonempty, sorted and unique")
        super().__init__(values, ids, lambda t: (ids[t].numel(), *t.default_factory().shape),
                         lambda t: t.__name__)

    @classmethod
    def make(cls, variables: Iterable[Var | VarWithValue]) -> VarValues:
        """Stack handles (default values) and handles with values by type,
        sorting each type's rows by ID."""
        ids_of, rows_of = defaultdict(list), defaultdict(list)
        for item in variables:
            var, value = (item.variable, item.value) if isinstance(item, VarWithValue) else (item, None)
            t, ids = type(var), as_ids(var.id)
            storage = t.default_factory().shape
            want = (*ids.shape, *storage)
            if value is None:
                value = t.default_factory().to(ids.device).expand(want)
            elif tuple(value.shape) != want:
                raise ValueError(f"{t.__name__}: expected shape {want}, got {tuple(value.shape)}")
            ids_of[t].append(ids.reshape(-1).cpu())
            rows_of[t].append(value.reshape(-1, *storage))
        values, ids = {}, {}
        for t in ids_of:
            all_ids, rows = torch.cat(ids_of[t]), torch.cat(rows_of[t])
            order = torch.argsort(all_ids)
            ids[t], values[t] = all_ids[order], rows[order.to(rows.device)]
        return cls(values, ids)

    def __getitem__(self, var):
        if isinstance(var, type):
            return self._values[var]
        want = as_ids(var.id).cpu()
        known = self._ids[type(var)]
        pos = torch.searchsorted(known, want).clamp_max(known.numel() - 1)
        if not torch.equal(known[pos], want):
            raise KeyError(f"Unknown {type(var).__name__} ID")
        return self._values[type(var)][pos.to(self.device)]

    def to(self, *args, **kwargs) -> VarValues:
        return VarValues({t: v.to(*args, **kwargs) for t, v in self._values.items()}, self._ids)

    def detach(self) -> VarValues:
        return VarValues({t: v.detach() for t, v in self._values.items()}, self._ids)

    def retract(self, tangent: Tensor, layout) -> VarValues:
        return VarValues(self._retracted(tangent, layout), self._ids)


__all__ = ["Parameterization", "ParameterRef", "Var", "VarValues", "VarWithValue", "VariableLayout",
           "NamedValues", "as_ids", "euclidean_type"]
