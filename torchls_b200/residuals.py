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


def sim3_log(pose: Tensor) -> Tensor:
    """Sim(3) logarithm -> [t(3), w(3), log s], inverse of ``sim3_exp``."""
    sr = pose[..., :3, :3]
    s = ((sr * sr).sum((-1, -2)) / 3).sqrt()
    sigma = s.log()
    w = so3_log(sr / s[..., None, None])
    # Translation part: t = W u, with W = sum_k (A)^k / (k+1)! for the
    # generator A = w^ + sigma I; solve W u = t via the closed-form W.
    wmat = sim3_left_jacobian(w, sigma)
    u = torch.linalg.solve(wmat, pose[..., :3, 3:4]).squeeze(-1)
    return torch.cat((u, w, sigma[..., None]), dim=-1)


def sim3_left_jacobian(w: Tensor, sigma: Tensor) -> Tensor:
    """W(w, sigma) = int_0^1 exp(s (w^ + sigma I)) ds, the Sim(3) 'V' matrix.

    Evaluated through ``torch.matrix_exp`` of the 4x4 block generator
    [[A, I], [0, 0]] whose top-right block equals W (exact for any A).
    """
    eye = torch.eye(3, dtype=w.dtype, device=w.device).expand(*w.shape[:-1], 3, 3)
    a = skew(w) + sigma[..., None, None] * eye
    zero = torch.zeros_like(a)
    big = torch.cat((torch.cat((a, eye), -1), torch.cat((zero, zero), -1)), -2)
    return torch.matrix_exp(big)[..., :3, 3:]


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

__all__ = ["camera_distance_prior", "point_prior", "reprojection", "se3_between", "sim3_between", "sim3_inverse", "sim3_log"]
