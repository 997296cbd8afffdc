"""Lie-group primitives in torch, usable inside torch.func transforms.

These are the user-facing forms of the retractions whose CUDA versions live in
``csrc/geometry.cuh``. Conventions follow torchls ``geometry.py``:

* SO(3) tangent: axis-angle (3).                     (torchls geometry.py:40-45)
* SE(3) tangent: [translation(3), rotation(3)].      (torchls geometry.py:48-57)
* Sim(3) tangent: [translation(3), rotation(3), log scale(1)]; the 3x3 block
  stores s*R.                                         (torchls geometry.py:60-73)
* Updates are right-multiplicative: X <- X * Exp(delta).
* The small-angle branch uses Taylor series when theta^2 < 1e-4
  (torchls geometry.py:19-37).
"""

from __future__ import annotations

import math

import torch
from torch import Tensor

from .variables import Var

SMALL_ANGLE2 = 1e-4


def skew(vector: Tensor) -> Tensor:
    """[v]x for (..., 3) vectors -> (..., 3, 3)."""
    x, y, z = vector.unbind(-1)
    o = torch.zeros_like(x)
    rows = (o, -z, y, z, o, -x, -y, x, o)
    return torch.stack(rows, dim=-1).reshape(*vector.shape[:-1], 3, 3)


def _rotation_series(rotation: Tensor):
    """Return A=sin(t)/t, B=(1-cos t)/t^2, C=(t-sin t)/t^3 with shape (..., 1, 1).

    Keeps a trailing singleton axis so broadcasting against 3x3 matrices works
    and float32 inputs stay float32 under forward-mode AD.
    """
    t2 = (rotation * rotation).sum(-1, keepdim=True)
    small = t2 < SMALL_ANGLE2
    safe_t2 = torch.where(small, torch.ones_like(t2), t2)
    t = safe_t2.sqrt()
    s, c = torch.sin(t), torch.cos(t)
    a_big = s / t
    b_big = (1 - c) / safe_t2
    c_big = (t - s) / (safe_t2 * t)
    t4 = t2 * t2
    a_small = 1 - t2 / 6 + t4 / 120
    b_small = 0.5 - t2 / 24 + t4 / 720
    c_small = 1.0 / 6 - t2 / 120 + t4 / 5040
    a = torch.where(small, a_small, a_big)
    b = torch.where(small, b_small, b_big)
    cc = torch.where(small, c_small, c_big)
    return a[..., None], b[..., None], cc[..., None]


def so3_exp(rotation: Tensor) -> Tensor:
    """Axis-angle (..., 3) -> rotation matrix (..., 3, 3) (Rodrigues)."""
    w = skew(rotation)
    a, b, _ = _rotation_series(rotation)
    eye = torch.eye(3, dtype=rotation.dtype, device=rotation.device)
    return eye + a * w + b * (w @ w)


def se3_exp(tangent: Tensor) -> Tensor:
    """SE(3) exponential of [t(3), w(3)] -> (..., 4, 4)."""
    t, w = tangent[..., :3], tangent[..., 3:6]
    W = skew(w)
    a, b, c = _rotation_series(w)
    eye = torch.eye(3, dtype=tangent.dtype, device=tangent.device)
    W2 = W @ W
    rot = eye + a * W + b * W2
    left = eye + b * W + c * W2
    top = torch.cat((rot, left @ t[..., None]), dim=-1)
    bottom = torch.zeros_like(top[..., :1, :])
    bottom[..., 0, 3] = 1
    return torch.cat((top, bottom), dim=-2)


def sim3_exp(tangent: Tensor) -> Tensor:
    """Sim(3) exponential of [t(3), w(3), log s] -> (..., 4, 4).

    Defined as the matrix exponential of [[w^ + sigma I, t], [0, 0]]; this
    torch form evaluates it with ``torch.matrix_exp``. The CUDA retraction
    uses a closed form that agrees with it to rounding.
    """
    eye = torch.eye(3, dtype=tangent.dtype, device=tangent.device)
    gen = skew(tangent[..., 3:6]) + tangent[..., 6:7, None] * eye
    top = torch.cat((gen, tangent[..., :3, None]), dim=-1)
    full = torch.cat((top, torch.zeros_like(top[..., :1, :])), dim=-2)
    return torch.matrix_exp(full)


def so3_retract_jvp(rotation: Tensor, direction: Tensor) -> Tensor:
    """d/d(delta) of R*Exp(delta) at 0, applied to ``direction``."""
    return rotation @ skew(direction)


def se3_retract_jvp(pose: Tensor, direction: Tensor) -> Tensor:
    """Storage-space differential of T*Exp(delta) at 0 (order [t, w])."""
    rot = pose[..., :3, :3]
    top = torch.cat((rot @ skew(direction[..., 3:6]), rot @ direction[..., :3, None]), dim=-1)
    return torch.cat((top, torch.zeros_like(top[..., :1, :])), dim=-2)


def sim3_retract_jvp(pose: Tensor, direction: Tensor) -> Tensor:
    """Storage-space differential of S*Exp(delta) at 0 (order [t, w, log s])."""
    sr = pose[..., :3, :3]
    block = sr @ skew(direction[..., 3:6]) + sr * direction[..., 6:7, None]
    top = torch.cat((block, sr @ direction[..., :3, None]), dim=-1)
    return torch.cat((top, torch.zeros_like(top[..., :1, :])), dim=-2)


def _se2_retract(pose: Tensor, delta: Tensor) -> Tensor:
    """SE(2) [x, y, angle] right update with the exact SE(2) exponential."""
    th = delta[2]
    small = th * th < SMALL_ANGLE2
    safe = torch.where(small, torch.ones_like(th), th)
    a = torch.where(small, 1 - th * th / 6, torch.sin(safe) / safe)
    b = torch.where(small, th / 2 - th * th * th / 24, (1 - torch.cos(safe)) / safe)
    lx = a * delta[0] - b * delta[1]
    ly = b * delta[0] + a * delta[1]
    c, s = torch.cos(pose[2]), torch.sin(pose[2])
    return torch.stack((pose[0] + c * lx - s * ly, pose[1] + s * lx + c * ly, pose[2] + th))


class SE2Var(Var, default_factory=lambda: torch.zeros(3), tangent_dim=3, retract_fn=_se2_retract):
    """SE(2) poses stored as [x, y, angle], updated on the right."""


class SE3Var(
    Var,
    default_factory=lambda: torch.eye(4),
    tangent_dim=6,
    retract_fn=lambda pose, delta: pose @ se3_exp(delta),
    retract_jvp_fn=se3_retract_jvp,
):
    """SE(3) 4x4 poses; right update with [translation(3), rotation(3)] tangent."""


class SO3Var(
    Var,
    default_factory=lambda: torch.eye(3),
    tangent_dim=3,
    retract_fn=lambda rotation, delta: rotation @ so3_exp(delta),
    retract_jvp_fn=so3_retract_jvp,
):
    """SO(3) 3x3 rotations; right update with an axis-angle tangent."""


class Sim3Var(
    Var,
    default_factory=lambda: torch.eye(4),
    tangent_dim=7,
    retract_fn=lambda pose, delta: pose @ sim3_exp(delta),
    retract_jvp_fn=sim3_retract_jvp,
):
    """Sim(3) 4x4 poses [sR, t; 0, 1], s > 0; tangent [t(3), w(3), log s]."""


# Tags read by the CUDA retraction: group kind per Var type.
SE3Var.cuda_kind = "se3"
SO3Var.cuda_kind = "so3"
Sim3Var.cuda_kind = "sim3"
SE2Var.cuda_kind = "se2"


def so3_log(rotation: Tensor) -> Tensor:
    """Rotation matrix -> axis-angle through a unit quaternion.

    Picks the numerically largest quaternion component, so the result is
    accurate near 0 and near pi; branch selection is tensor-only and works
    under vmap/jacrev.
    """
    m = rotation
    r00, r11, r22 = m[..., 0, 0], m[..., 1, 1], m[..., 2, 2]
    trace_terms = torch.stack(
        (1 + r00 + r11 + r22, 1 + r00 - r11 - r22, 1 - r00 + r11 - r22, 1 - r00 - r11 + r22), -1
    )
    mag = trace_terms.clamp_min(1e-12).sqrt()
    d21, d02, d10 = m[..., 2, 1] - m[..., 1, 2], m[..., 0, 2] - m[..., 2, 0], m[..., 1, 0] - m[..., 0, 1]
    s01, s02, s12 = m[..., 0, 1] + m[..., 1, 0], m[..., 0, 2] + m[..., 2, 0], m[..., 1, 2] + m[..., 2, 1]
    cand = torch.stack(
        (
            torch.stack((mag[..., 0] ** 2, d21, d02, d10), -1),
            torch.stack((d21, mag[..., 1] ** 2, s01, s02), -1),
            torch.stack((d02, s01, mag[..., 2] ** 2, s12), -1),
            torch.stack((d10, s02, s12, mag[..., 3] ** 2), -1),
        ),
        -2,
    ) / (2 * mag[..., :, None])
    pick = mag.argmax(-1)[..., None, None].expand(*mag.shape[:-1], 1, 4)
    q = cand.gather(-2, pick).squeeze(-2)
    q = torch.where(q[..., :1] < 0, -q, q)
    vec = q[..., 1:]
    n = (vec * vec).sum(-1, keepdim=True).clamp_min(1e-24).sqrt()
    angle = 2 * torch.atan2(n, q[..., :1])
    return vec * (angle / n)


def se3_log(pose: Tensor) -> Tensor:
    """SE(3) logarithm -> [t(3), w(3)], inverse of :func:`se3_exp`."""
    w = so3_log(pose[..., :3, :3])
    W = skew(w)
    t2 = (w * w).sum(-1, keepdim=True)
    # V^-1 = I - W/2 + k W^2, k = (1 - (t/2) cot(t/2)) / t^2; the closed form
    # cancels for small t, so a Taylor series is used below t = 0.5.
    small = t2 < 0.25
    safe_t2 = torch.where(small, torch.ones_like(t2), t2)
    half = safe_t2.sqrt() / 2
    k_big = (1 - half * torch.cos(half) / torch.sin(half)) / safe_t2
    k_small = 1.0 / 12 + t2 * (1.0 / 720 + t2 * (1.0 / 30240 + t2 * (1.0 / 1209600 + t2 / 47900160)))
    k = torch.where(small, k_small, k_big)[..., None]
    eye = torch.eye(3, dtype=pose.dtype, device=pose.device)
    vinv = eye - 0.5 * W + k * (W @ W)
    u = (vinv @ pose[..., :3, 3:4]).squeeze(-1)
    return torch.cat((u, w), dim=-1)


def se3_inverse(pose: Tensor) -> Tensor:
    rt = pose[..., :3, :3].transpose(-1, -2)
    top = torch.cat((rt, -(rt @ pose[..., :3, 3:4])), dim=-1)
    return torch.cat((top, pose[..., 3:4, :]), dim=-2)


__all__ = [
    "SE2Var",
    "SE3Var",
    "SO3Var",
    "Sim3Var",
    "se3_exp",
    "se3_inverse",
    "se3_log",
    "se3_retract_jvp",
    "sim3_exp",
    "sim3_retract_jvp",
    "skew",
    "so3_exp",
    "so3_log",
    "so3_retract_jvp",
]
