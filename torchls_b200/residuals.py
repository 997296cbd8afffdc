"""Built-in residual functions with fused CUDA linearization kernels.

Each function is an ordinary single-observation torch residual (so it works
under ``torch.func`` and with torchls itself); its ``cuda_residual`` tag tells
the CUDA backend to evaluate the residual and its analytic Jacobian with one
fused kernel instead of ``vmap(jacrev(...))``.
"""

from __future__ import annotations

import torch
from torch import Tensor

from .geometry import se3_inverse, se3_log, skew, so3_log

DEPTH_EPS = 1e-6


def reprojection(camera: Tensor, point: Tensor, observation: Tensor) -> Tensor:
    """Normalized pinhole reprojection error with a depth guard.

    ``camera`` is a world-to-camera 4x4 pose, ``point`` a world 3-vector,
    ``observation`` normalized image coordinates (2). Points at depth
    z <= 1e-6 give a zero residual and zero derivatives (torchls README.md:22-34).
    """
    xyz = camera[:3, :3] @ point + camera[:3, 3]
    valid = xyz[2] > DEPTH_EPS
    z = torch.where(valid, xyz[2], torch.ones_like(xyz[2]))
    err = xyz[:2] / z - observation
    return torch.where(valid, err, torch.zeros_like(err))


def se3_between(pose_i: Tensor, pose_j: Tensor, measurement: Tensor) -> Tensor:
    """Relative-pose error log(Z^-1 T_i^-1 T_j) in [t, w] order (6)."""
    return se3_log(se3_inverse(measurement) @ se3_inverse(pose_i) @ pose_j)


def sim3_inverse(pose: Tensor) -> Tensor:
    sr = pose[..., :3, :3]
    s2 = (sr * sr).sum((-1, -2), keepdim=True) / 3
    inv_sr = sr.transpose(-1, -2) / s2
    top = torch.cat((inv_sr, -(inv_sr @ pose[..., :3, 3:4])), dim=-1)
    return torch.cat((top, pose[..., 3:4, :]), dim=-2)


def sim3_w_coefficients(sigma: Tensor, t2: Tensor):
    """Coefficients of W(w, sigma) = int_0^1 exp(s (w^ + sigma I)) ds = a0 I + c1 w^ + c2 w^2.

    With z = sigma + i theta (theta^2 = |w|^2 = t2) and F = (e^z - 1) / z:
    a0 = (e^sigma - 1) / sigma, c1 = Im F / theta, c2 = (a0 - Re F) / theta^2.
    Where |z| <= 4, or theta^2 < 1e-2 and |sigma| <= 10, the entire series
    F = sum_k z^k / (k+1)! is summed in (sigma, theta^2) by the recurrences
    z^k = a_k + i theta b_k, c_k = (sigma^k - a_k) / theta^2 (64 terms); elsewhere
    the closed forms (theta^2 >= 1e-2 there, so they cancel by at most 100x).
    Tensor-only, so it works under vmap / jacrev; the CUDA between-factor
    kernel evaluates the same formulas.
    """
    z2 = sigma * sigma + t2
    series = (z2 <= 16.0) | ((t2 < 1e-2) & (sigma * sigma <= 100.0))
    # series with inputs kept small where it is not selected (no inf/nan in either branch)
    ss = torch.where(series, sigma, torch.zeros_like(sigma))
    st = torch.where(series, t2, torch.zeros_like(t2))
    a, b, c, sp = torch.ones_like(ss), torch.zeros_like(ss), torch.zeros_like(ss), torch.ones_like(ss)
    sa, sb, sc = torch.zeros_like(ss), torch.zeros_like(ss), torch.zeros_like(ss)
    inv = 1.0
    for k in range(64):
        inv = inv / (k + 1)
        sa, sb, sc = sa + inv * sp, sb + inv * b, sc + inv * c
        a, b, c = ss * a - st * b, a + ss * b, ss * c + b
        sp = sp * ss
    # closed forms with inputs kept away from 0 where they are not selected
    cs_ = torch.where(series, torch.full_like(sigma, 3.0), sigma)
    ct = torch.where(series, torch.ones_like(t2), t2)
    th, es = ct.sqrt(), torch.exp(cs_)
    den = cs_ * cs_ + ct
    a0c = (es - 1) / cs_
    ref = (cs_ * (es * torch.cos(th) - 1) + th * es * torch.sin(th)) / den
    imf = (cs_ * es * torch.sin(th) - th * (es * torch.cos(th) - 1)) / den
    return (torch.where(series, sa, a0c), torch.where(series, sb, imf / th),
            torch.where(series, sc, (a0c - ref) / ct))


def sim3_left_jacobian(w: Tensor, sigma: Tensor) -> Tensor:
    """W(w, sigma) = int_0^1 exp(s (w^ + sigma I)) ds, the Sim(3) 'V' matrix."""
    a0, c1, c2 = sim3_w_coefficients(sigma, (w * w).sum(-1))
    W = skew(w)
    eye = torch.eye(3, dtype=w.dtype, device=w.device)
    return a0[..., None, None] * eye + c1[..., None, None] * W + c2[..., None, None] * (W @ W)


def _solve3(M: Tensor, t: Tensor) -> Tensor:
    """M^-1 t for 3x3 M by the adjugate (tensor-only; no batched LAPACK call)."""
    c0 = torch.linalg.cross(M[..., 1, :], M[..., 2, :])
    c1 = torch.linalg.cross(M[..., 2, :], M[..., 0, :])
    c2 = torch.linalg.cross(M[..., 0, :], M[..., 1, :])
    det = (M[..., 0, :] * c0).sum(-1)
    adj = torch.stack((c0, c1, c2), -1)  # columns are the cofactor rows
    return (adj @ t[..., None]).squeeze(-1) / det[..., None]


def sim3_log(pose: Tensor) -> Tensor:
    """Sim(3) logarithm -> [t(3), w(3), log s], inverse of ``sim3_exp``:
    s = sqrt(|sR|_F^2 / 3), w = so3_log(sR / s), t = W(w, log s) u."""
    sr = pose[..., :3, :3]
    s = ((sr * sr).sum((-1, -2)) / 3).sqrt()
    sigma = s.log()
    w = so3_log(sr / s[..., None, None])
    u = _solve3(sim3_left_jacobian(w, sigma), pose[..., :3, 3])
    return torch.cat((u, w, sigma[..., None]), dim=-1)


def sim3_between(pose_i: Tensor, pose_j: Tensor, measurement: Tensor) -> Tensor:
    """Relative similarity error log(Z^-1 S_i^-1 S_j) (7)."""
    return sim3_log(sim3_inverse(measurement) @ sim3_inverse(pose_i) @ pose_j)


def point_prior(point: Tensor, reference: Tensor) -> Tensor:
    return point - reference


reprojection.cuda_residual = "reprojection"
def camera_distance_prior(camera: Tensor, reference: Tensor, distance: Tensor) -> Tensor:
    """|c - c_ref| - distance for world-to-camera poses (c = -R^T t): fixes the
    global scale of a bundle adjustment whose first camera is held fixed."""
    c = -(camera[:3, :3].transpose(-1, -2) @ camera[:3, 3])
    c0 = -(reference[:3, :3].transpose(-1, -2) @ reference[:3, 3])
    return (torch.linalg.vector_norm(c - c0) - distance).reshape(1)


se3_between.cuda_residual = "se3_between"
sim3_between.cuda_residual = "sim3_between"

__all__ = ["camera_distance_prior", "point_prior", "reprojection", "se3_between", "sim3_between", "sim3_inverse",
           "sim3_left_jacobian", "sim3_log"]
