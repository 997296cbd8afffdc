"""Lie-group maps in numpy (float64). Restates torchls geometry.py:10-107.

Tangent orders: SE(3) [t, w]; Sim(3) [t, w, log s]; right updates X*Exp(d).
Small-angle Taylor branch below theta^2 = 1e-4 (geometry.py:19-37).
"""

from __future__ import annotations

import numpy as np
from scipy.linalg import expm


def skew(v):
    v = np.asarray(v, dtype=np.float64)
    out = np.zeros(v.shape[:-1] + (3, 3))
    out[..., 0, 1], out[..., 0, 2] = -v[..., 2], v[..., 1]
    out[..., 1, 0], out[..., 1, 2] = v[..., 2], -v[..., 0]
    out[..., 2, 0], out[..., 2, 1] = -v[..., 1], v[..., 0]
    return out


def rotation_coefficients(w):
    """sin t / t, (1 - cos t)/t^2, (t - sin t)/t^3 (geometry.py:19-37)."""
    t2 = np.sum(w * w, axis=-1)
    small = t2 < 1e-4
    t = np.sqrt(np.where(small, 1.0, t2))
    a = np.where(small, 1 - t2 / 6 + t2**2 / 120, np.sin(t) / t)
    b = np.where(small, 0.5 - t2 / 24 + t2**2 / 720, (1 - np.cos(t)) / np.where(small, 1.0, t2))
    c = np.where(small, 1 / 6 - t2 / 120 + t2**2 / 5040, (t - np.sin(t)) / (t**3))
    return a[..., None, None], b[..., None, None], c[..., None, None]


def so3_exp(w):
    W = skew(w)
    a, b, _ = rotation_coefficients(w)
    return np.eye(3) + a * W + b * (W @ W)


def se3_exp(xi):
    """geometry.py:48-57."""
    xi = np.asarray(xi, dtype=np.float64)
    t, w = xi[..., :3], xi[..., 3:6]
    W = skew(w)
    a, b, c = rotation_coefficients(w)
    W2 = W @ W
    out = np.zeros(xi.shape[:-1] + (4, 4))
    out[..., :3, :3] = np.eye(3) + a * W + b * W2
    out[..., :3, 3] = ((np.eye(3) + b * W + c * W2) @ t[..., None])[..., 0]
    out[..., 3, 3] = 1
    return out


def sim3_exp(xi):
    """Matrix exponential of the Sim(3) generator (geometry.py:60-73)."""
    xi = np.asarray(xi, dtype=np.float64)
    gen = np.zeros(xi.shape[:-1] + (4, 4))
    gen[..., :3, :3] = skew(xi[..., 3:6]) + xi[..., 6, None, None] * np.eye(3)
    gen[..., :3, 3] = xi[..., :3]
    flat = gen.reshape(-1, 4, 4)
    return np.stack([expm(m) for m in flat]).reshape(gen.shape)


def se2_retract(pose, delta):
    th = delta[..., 2]
    small = th * th < 1e-4
    safe = np.where(small, 1.0, th)
    a = np.where(small, 1 - th * th / 6, np.sin(safe) / safe)
    b = np.where(small, th / 2 - th**3 / 24, (1 - np.cos(safe)) / safe)
    lx = a * delta[..., 0] - b * delta[..., 1]
    ly = b * delta[..., 0] + a * delta[..., 1]
    c, s = np.cos(pose[..., 2]), np.sin(pose[..., 2])
    return np.stack((pose[..., 0] + c * lx - s * ly, pose[..., 1] + s * lx + c * ly, pose[..., 2] + th), -1)


def retract(kind, values, delta):
    """Right retraction per group kind (variables.py:153-160, geometry.py:110-160)."""
    if kind == "euclidean":
        return values + delta.reshape(values.shape)
    if kind == "se3":
        return values @ se3_exp(delta)
    if kind == "so3":
        return values @ so3_exp(delta)
    if kind == "sim3":
        return values @ sim3_exp(delta)
    if kind == "se2":
        return se2_retract(values, delta)
    raise ValueError(f"oracle has no retraction for {kind!r}")


def so3_log(R):
    """Rotation -> axis-angle via the largest quaternion component (Shepperd)."""
    R = np.asarray(R, dtype=np.float64)
    tr = np.stack(
        (
            1 + R[..., 0, 0] + R[..., 1, 1] + R[..., 2, 2],
            1 + R[..., 0, 0] - R[..., 1, 1] - R[..., 2, 2],
            1 - R[..., 0, 0] + R[..., 1, 1] - R[..., 2, 2],
            1 - R[..., 0, 0] - R[..., 1, 1] + R[..., 2, 2],
        ),
        -1,
    )
    mag = np.sqrt(np.maximum(tr, 1e-12))
    k = np.argmax(mag, axis=-1)
    d21, d02, d10 = R[..., 2, 1] - R[..., 1, 2], R[..., 0, 2] - R[..., 2, 0], R[..., 1, 0] - R[..., 0, 1]
    s01, s02, s12 = R[..., 0, 1] + R[..., 1, 0], R[..., 0, 2] + R[..., 2, 0], R[..., 1, 2] + R[..., 2, 1]
    cand = np.stack(
        (
            np.stack((mag[..., 0] ** 2, d21, d02, d10), -1),
            np.stack((d21, mag[..., 1] ** 2, s01, s02), -1),
            np.stack((d02, s01, mag[..., 2] ** 2, s12), -1),
            np.stack((d10, s02, s12, mag[..., 3] ** 2), -1),
        ),
        -2,
    ) / (2 * mag[..., :, None])
    q = np.take_along_axis(cand, k[..., None, None].repeat(4, -1), axis=-2)[..., 0, :]
    q = np.where(q[..., :1] < 0, -q, q)
    n = np.sqrt(np.maximum(np.sum(q[..., 1:] ** 2, -1, keepdims=True), 1e-24))
    return q[..., 1:] * (2 * np.arctan2(n, q[..., :1]) / n)
