"""Problem model, linearization, losses and trial costs (numpy, float64).

Restates:
* layout in declaration order, offset += count*dim        (named.py:86-119)
* ID -> row (searchsorted) and global columns            (problem.py:66-74, 138-148)
* weights as float64, data broadcasting / in_dims          (problem.py:83-103, 201-221)
* linearization at delta=0 through the retraction chart    (linearization.py:62-112)
* robust losses: Huber scaling, generic Triggs correction,
  divided-difference reductions                            (losses.py:13-107)
* cost, residuals, exact trial reduction                   (problem.py:292-348)
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import geometry


# ----------------------------------------------------------------------------- losses
@dataclass(frozen=True)
class huber_loss:
    """Huber on a block's squared norm s (losses.py:56-107)."""

    delta: float

    def evaluate(self, s):
        tiny = np.finfo(np.float64).tiny
        safe = np.maximum(s, tiny)
        norm = np.sqrt(safe)
        out = s > self.delta * self.delta
        first = np.where(out, self.delta / norm, 1.0)
        value = np.where(out, self.delta * (2 * norm - self.delta), s)
        second = np.where(out, -0.5 * first / safe, 0.0)
        return value, first, second

    def value(self, s):
        norm = np.sqrt(np.maximum(s, np.finfo(np.float64).tiny))
        return np.where(s > self.delta * self.delta, self.delta * (2 * norm - self.delta), s)

    def linearize(self, residual, blocks, s, evaluation):
        w = np.sqrt(evaluation[1])
        return residual * w[:, None], [b * w[:, None, None] for b in blocks]

    def reduction(self, before, after, sqdiff):
        """Divided difference of rho (losses.py:92-107)."""
        tiny = np.finfo(np.float64).tiny
        a, b = np.sqrt(before), np.sqrt(after)
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        short = np.maximum(self.delta - lo, 0.0)
        crossing = (2 * self.delta - short * (short / np.maximum(hi - lo, tiny))) / np.maximum(a + b, tiny)
        coef = np.where(
            hi <= self.delta,
            1.0,
            np.where(lo >= self.delta, 2 * self.delta / np.maximum(a + b, tiny), crossing),
        )
        return sqdiff * coef


class generic_loss:
    """A loss given by evaluate(s) -> (rho, rho', rho''); Triggs/Ceres correction (losses.py:30-53)."""

    def __init__(self, evaluate):
        self._evaluate = evaluate

    def evaluate(self, s):
        return self._evaluate(s)

    def value(self, s):
        return self._evaluate(s)[0]

    def linearize(self, residual, blocks, s, evaluation):
        _, first, second = evaluation
        tiny = np.finfo(np.float64).tiny
        positive = (s > 0) & (second > 0)
        ratio = np.where(positive, 2 * s * second / np.maximum(first, tiny), 0.0)
        alpha = -ratio / (1 + np.sqrt(1 + ratio))
        corr = alpha / np.maximum(s, tiny)
        w = np.sqrt(first)
        out = []
        for b in blocks:
            rtj = np.einsum("nr,nrd->nd", residual, b)
            out.append(w[:, None, None] * (b - corr[:, None, None] * residual[:, :, None] * rtj[:, None, :]))
        return residual * (w / (1 - alpha))[:, None], out

    def reduction(self, before, after, sqdiff):
        return self.value(before) - self.value(after)


# ----------------------------------------------------------------------------- residuals
def reprojection_with_jacobian(camera, point, uv, *, cam_var, point_var):
    """Analytic residual and Jacobians of the depth-guarded reprojection.

    d xyz / d[t, w] = [R, -R [p]x] under the right SE(3) chart
    (geometry.py:92-107); d xyz / d p = R.
    """
    R, t = camera[:, :3, :3], camera[:, :3, 3]
    xyz = np.einsum("nij,nj->ni", R, point) + t
    valid = xyz[:, 2] > 1e-6
    z = np.where(valid, xyz[:, 2], 1.0)
    r = xyz[:, :2] / z[:, None] - uv
    r = np.where(valid[:, None], r, 0.0)
    dproj = np.zeros((len(z), 2, 3))
    dproj[:, 0, 0] = 1 / z
    dproj[:, 1, 1] = 1 / z
    dproj[:, 0, 2] = -xyz[:, 0] / z**2
    dproj[:, 1, 2] = -xyz[:, 1] / z**2
    dproj = np.where(valid[:, None, None], dproj, 0.0)
    blocks = []
    if cam_var:
        dxyz = np.concatenate((R, -R @ geometry.skew(point)), axis=-1)
        blocks.append(dproj @ dxyz)
    if point_var:
        blocks.append(dproj @ R)
    return r, blocks


def _torch_jvp(kind):
    import torch

    if kind == "euclidean":
        return lambda x, d: x + d.reshape(x.shape)

    def hat(v):
        x, y, z = v.unbind(-1)
        o = torch.zeros_like(x)
        return torch.stack((o, -z, y, z, o, -x, -y, x, o), -1).reshape(*v.shape[:-1], 3, 3)

    if kind == "so3":
        return lambda R, d: R + R @ hat(d)
    if kind == "se3":
        def f(T, d):
            top = torch.cat((T[:3, :3] @ hat(d[3:6]), (T[:3, :3] @ d[:3])[:, None]), -1)
            return T + torch.cat((top, torch.zeros_like(top[:1])), 0)
        return f
    if kind == "sim3":
        def f(S, d):
            sr = S[:3, :3]
            top = torch.cat((sr @ hat(d[3:6]) + sr * d[6], (sr @ d[:3])[:, None]), -1)
            return S + torch.cat((top, torch.zeros_like(top[:1])), 0)
        return f
    return None


def autodiff_linearize(fn, args, var_positions, kinds, dims):
    """vmap(jacrev) of fn through the first-order retraction chart at delta=0
    (linearization.py:67-96), on CPU in float64."""
    import torch

    targs = [torch.as_tensor(a, dtype=torch.float64) if np.asarray(a).dtype.kind == "f"
             else torch.as_tensor(a) for a in args]
    jvps = [_torch_jvp(k) for k in kinds]

    def local(deltas, *xs):
        xs = list(xs)
        for pos, jvp, d in zip(var_positions, jvps, deltas):
            xs[pos] = jvp(xs[pos], d)
        out = fn(*xs).reshape(-1)
        return out, out

    zeros = tuple(torch.zeros(d, dtype=torch.float64) for d in dims)
    jac = torch.func.vmap(torch.func.jacrev(local, argnums=0, has_aux=True),
                          in_dims=(None, *([0] * len(targs))))
    blocks, res = jac(zeros, *targs)
    return res.numpy(), [b.numpy() for b in blocks]


# ----------------------------------------------------------------------------- problem
@dataclass
class Group:
    key: str
    kind: str
    values: np.ndarray
    offset: int

    @property
    def count(self):
        return self.values.shape[0]

    @property
    def dim(self):
        if self.kind == "euclidean":
            return int(np.prod(self.values.shape[1:]))
        return {"se3": 6, "so3": 3, "sim3": 7, "se2": 3}[self.kind]


@dataclass
class Batch:
    fn: object
    args: list  # ("var", group, rows[N]) or ("data", array[N,...] or shared)
    count: int
    loss: object
    weights: np.ndarray | None
    slots: list  # argument positions that are variables
    groups: list  # group index per slot
    rows: list  # row indices per slot


class OracleProblem:
    """``Problem``-style container (named.py:24-154) for the oracle."""

    def __init__(self, parameters: dict, manifolds: dict | None = None):
        manifolds = manifolds or {}
        self.groups = []
        offset = 0
        for key, value in parameters.items():
            value = np.asarray(value, dtype=np.float64)
            g = Group(key, manifolds.get(key, "euclidean"), value.copy(), offset)
            self.groups.append(g)
            offset += g.count * g.dim
        self.tangent_dim = offset
        self.batches: list[Batch] = []
        self.index = {g.key: i for i, g in enumerate(self.groups)}

    def add_residual(self, fn, *args, in_dims=None, loss=None, weights=None):
        refs = [a for a in args if isinstance(a, tuple)]
        batched = [np.asarray(a[1]).size for a in refs if np.ndim(a[1]) == 1]
        count = max(batched, default=1)
        out_args, slots, groups, rows = [], [], [], []
        for pos, a in enumerate(args):
            if isinstance(a, tuple):
                r = np.broadcast_to(np.asarray(a[1], dtype=np.int64).reshape(-1), (count,)).copy()
                gi = self.index[a[0]]
                out_args.append(("var", gi, r))
                slots.append(pos)
                groups.append(gi)
                rows.append(r)
            else:
                arr = np.asarray(a)
                if arr.dtype.kind == "f":
                    arr = arr.astype(np.float64)
                axis = None if in_dims is None else in_dims[pos]
                if in_dims is None:
                    axis = 0 if batched and arr.ndim > 0 else None
                if axis is None:
                    arr = np.broadcast_to(arr[None], (count, *arr.shape))
                else:
                    arr = np.broadcast_to(arr, (count, *arr.shape[1:]))
                out_args.append(("data", arr))
        w = None
        if weights is not None:
            w = np.broadcast_to(np.asarray(weights, dtype=np.float64).reshape(-1), (count,)).copy()
        self.batches.append(Batch(fn, out_args, count, loss, w, slots, groups, rows))
        return self

    @property
    def has_loss(self):
        return any(b.loss is not None or b.weights is not None for b in self.batches)

    # -- values
    def values(self):
        return [g.values.copy() for g in self.groups]

    def gather(self, batch, values):
        out = []
        for a in batch.args:
            out.append(values[a[1]][a[2]] if a[0] == "var" else a[1])
        return out

    def columns(self, batch, slot):
        g = self.groups[batch.groups[slot]]
        return batch.rows[slot][:, None] * g.dim + g.offset + np.arange(g.dim)[None, :]

    def retract(self, values, delta):
        out = []
        for g, v in zip(self.groups, values):
            d = delta[g.offset : g.offset + g.count * g.dim].reshape(g.count, g.dim)
            out.append(geometry.retract(g.kind, v, d))
        return out

    # -- residual evaluation
    def _raw(self, batch, values, with_jacobian):
        args = self.gather(batch, values)
        tag = getattr(batch.fn, "cuda_residual", None)
        kinds = [self.groups[g].kind for g in batch.groups]
        if tag == "reprojection" and all(k in ("se3", "euclidean") for k in kinds):
            cam_var = 0 in batch.slots
            pt_var = 1 in batch.slots
            if (not cam_var or self.groups[batch.groups[0]].kind == "se3"):
                r, blocks = reprojection_with_jacobian(args[0], args[1], args[2],
                                                       cam_var=cam_var, point_var=pt_var)
                return r, blocks
        if not with_jacobian:
            import torch

            targs = [torch.as_tensor(np.ascontiguousarray(a)) for a in args]
            r = torch.func.vmap(batch.fn)(*targs)
            return r.reshape(batch.count, -1).numpy(), None
        dims = [self.groups[g].dim for g in batch.groups]
        return autodiff_linearize(batch.fn, [np.ascontiguousarray(a) for a in args],
                                  batch.slots, kinds, dims)

    def residuals(self, values):
        """Raw residuals, observation-major, batches concatenated (problem.py:292-299)."""
        return np.concatenate([self._raw(b, values, False)[0].reshape(-1) for b in self.batches])

    def cost(self, values):
        """problem.py:301-313."""
        if not self.has_loss:
            return 0.5 * float(np.sum(self.residuals(values) ** 2))
        total = 0.0
        for b in self.batches:
            r = self._raw(b, values, False)[0]
            s = np.sum(r * r, -1)
            v = s if b.loss is None else b.loss.value(s)
            total += float(np.sum(v if b.weights is None else b.weights * v))
        return 0.5 * total

    def linearize(self, values):
        """Linearization (problem.py:350-368, 157-183; linearization.py:91-112)."""
        groups, res, raws, objective = [], [], [], 0.0
        for b in self.batches:
            r, blocks = self._raw(b, values, True)
            raw = r
            if self.has_loss:
                s = np.sum(r * r, -1)
                if b.loss is None:
                    obj = s
                else:
                    ev = b.loss.evaluate(s)
                    obj = ev[0]
                    r, blocks = b.loss.linearize(r, blocks, s, ev)
                if b.weights is not None:
                    sw = np.sqrt(b.weights)
                    r = r * sw[:, None]
                    blocks = [blk * sw[:, None, None] for blk in blocks]
                    obj = obj * b.weights
                objective += float(np.sum(obj))
                raws.append(raw.reshape(-1))
            res.append(r.reshape(-1))
            groups.append(
                dict(
                    blocks=[np.ascontiguousarray(x) for x in blocks],
                    columns=[self.columns(b, s) for s in range(len(b.slots))],
                    types=list(b.groups),
                    rows=list(b.rows),
                )
            )
        residual = np.concatenate(res)
        from .linalg import BlockJacobian

        J = BlockJacobian(groups, self.groups, (residual.size, self.tangent_dim))
        cost = 0.5 * objective if self.has_loss else 0.5 * float(np.sum(residual**2))
        return Linearization(residual, J, np.concatenate(raws) if self.has_loss else None, cost)

    def evaluate_trial(self, values, lin):
        """Objective and exact reduction at a proposed point (problem.py:315-348)."""
        proposed = self.residuals(values)
        if not self.has_loss:
            before = lin.residual
            return 0.5 * float(np.sum(proposed**2)), 0.5 * float(np.dot(before - proposed, before + proposed))
        objs, reds, off = 0.0, 0.0, 0
        for k, b in enumerate(self.batches):
            n = b.count
            rdim = lin.jacobian.groups[k]["blocks"][0].shape[1]
            old = lin.raw_residual[off : off + n * rdim].reshape(n, rdim)
            new = proposed[off : off + n * rdim].reshape(n, rdim)
            off += n * rdim
            so, sn = np.sum(old * old, -1), np.sum(new * new, -1)
            diff = np.sum((old - new) * (old + new), -1)
            val = sn if b.loss is None else b.loss.value(sn)
            red = diff if b.loss is None else b.loss.reduction(so, sn, diff)
            objs += float(np.sum(val if b.weights is None else b.weights * val))
            reds += float(np.sum(red if b.weights is None else b.weights * red))
        return 0.5 * objs, 0.5 * reds


@dataclass
class Linearization:
    residual: np.ndarray
    jacobian: object
    raw_residual: np.ndarray | None
    cost: float

    @property
    def gradient(self):
        return self.jacobian.rmatvec(self.residual)
