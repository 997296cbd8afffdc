"""Seeded synthetic problems: bundle adjustment and SE(3) pose graphs.

There is no public dataset for these workloads; every problem is generated on
the CPU from a ``torch.Generator`` seed, in float64, and then moved to the
requested device. The same arrays feed the CUDA solver, the CPU oracle and the
reference implementation.

Bundle adjustment (``make_bundle_adjustment``)
    Cameras: ``num_cameras`` world-to-camera SE(3) poses at angle 2*pi*k/C on
    a circle of radius ``radius`` at height ``height``, looking at the origin
    (rows x, y, z of R; z = -c/|c|, x = z cross (0,0,1), y = z cross x).
    Points: uniform in [-1, 1]^3. Each point is observed by ``views`` distinct
    cameras chosen uniformly from the candidates (all cameras, or those within
    ``azimuth_window`` radians of the point's azimuth). Observations are
    point-major. uv = normalized pinhole projection + N(0, noise^2).
    Initial values: T0 = T * se3_exp([N(0, tn^2)^3, N(0, rn^2)^3]),
    P0 = P + N(0, pn^2). Camera 0 is held fixed: it is constant data for its
    observations and the optimised group holds cameras 1..C-1.

Pose graph (``make_pose_graph``)
    A 3D random walk of unit steps with yaw increments N(0, yaw^2) and a small
    vertical drift. Odometry edges (i, i+1) plus loop edges sampled uniformly
    with replacement among pose pairs (i, j), j > i + 1, with |p_i - p_j| <= 3.
    Measurements Z = T_i^-1 T_j * se3_exp(noise); initial poses integrate the
    noisy odometry; pose 0 is held fixed (constant data for its edges).

Sim(3) pose graph (``make_sim3_pose_graph``)
    The same walk and edge rule with a scale drift: pose k stores
    [s_k R_k, t_k; 0, 1], log s_k a random walk of N(0, scale_sigma^2) steps.
    Measurements Z = S_i^-1 S_j * sim3_exp([N(0, tn^2)^3, N(0, rn^2)^3,
    N(0, sn^2)]); initial poses integrate the noisy odometry; pose 0 fixed.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch
from torch import Tensor

from .geometry import se3_exp, se3_inverse, sim3_exp


@dataclass
class BundleAdjustmentData:
    cameras_true: Tensor  # [C, 4, 4]
    points_true: Tensor  # [P, 3]
    cameras_init: Tensor  # [C, 4, 4]
    points_init: Tensor  # [P, 3]
    camera_index: Tensor  # [M] int64
    point_index: Tensor  # [M] int64
    uv: Tensor  # [M, 2]

    @property
    def num_observations(self) -> int:
        return int(self.camera_index.numel())

    def split_fixed_camera(self):
        """Return (free-camera obs mask, camera-0 obs mask)."""
        fixed = self.camera_index == 0
        return ~fixed, fixed


def look_at_cameras(num_cameras: int, radius: float = 5.0, height: float = 1.0) -> Tensor:
    angles = torch.arange(num_cameras, dtype=torch.float64) * (2 * math.pi / num_cameras)
    centers = torch.stack(
        (radius * angles.cos(), radius * angles.sin(), torch.full_like(angles, height)), -1
    )
    z = -centers / centers.norm(dim=-1, keepdim=True)
    up = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64).expand_as(z)
    x = torch.linalg.cross(z, up)
    x = x / x.norm(dim=-1, keepdim=True)
    y = torch.linalg.cross(z, x)
    rot = torch.stack((x, y, z), dim=-2)
    trans = -(rot @ centers[..., None]).squeeze(-1)
    poses = torch.eye(4, dtype=torch.float64).repeat(num_cameras, 1, 1)
    poses[:, :3, :3] = rot
    poses[:, :3, 3] = trans
    return poses


def project(poses: Tensor, points: Tensor) -> Tensor:
    local = (poses[..., :3, :3] @ points[..., None]).squeeze(-1) + poses[..., :3, 3]
    return local[..., :2] / local[..., 2:3]


def make_bundle_adjustment(
    num_cameras: int = 10,
    num_points: int = 500,
    views: int = 8,
    *,
    seed: int = 0,
    azimuth_window: float | None = None,
    noise: float = 1e-3,
    translation_noise: float = 0.05,
    rotation_noise: float = 0.01,
    point_noise: float = 0.05,
    radius: float = 5.0,
    height: float = 1.0,
) -> BundleAdjustmentData:
    """Generate one seeded bundle-adjustment problem (float64, CPU)."""
    if views > num_cameras:
        raise ValueError("views must not exceed num_cameras")
    g = torch.Generator().manual_seed(seed)
    cams = look_at_cameras(num_cameras, radius, height)
    pts = torch.rand(num_points, 3, generator=g, dtype=torch.float64) * 2 - 1
    keys = torch.rand(num_points, num_cameras, generator=g, dtype=torch.float64)
    if azimuth_window is not None:
        cam_angle = torch.arange(num_cameras, dtype=torch.float64) * (2 * math.pi / num_cameras)
        pt_angle = torch.atan2(pts[:, 1], pts[:, 0])
        diff = torch.remainder(cam_angle[None, :] - pt_angle[:, None] + math.pi, 2 * math.pi) - math.pi
        allowed = diff.abs() <= azimuth_window
        if bool((allowed.sum(-1) < views).any()):
            raise ValueError("azimuth window leaves fewer candidate cameras than views")
        keys = torch.where(allowed, keys, torch.full_like(keys, 2.0))
    # A uniformly random subset of the allowed cameras: the `views` smallest keys.
    chosen = keys.topk(views, dim=-1, largest=False).indices
    cam_idx = chosen.reshape(-1)
    pt_idx = torch.arange(num_points).repeat_interleave(views)
    uv = project(cams[cam_idx], pts[pt_idx])
    uv = uv + noise * torch.randn(uv.shape, generator=g, dtype=torch.float64)
    perturb = torch.cat(
        (
            translation_noise * torch.randn(num_cameras, 3, generator=g, dtype=torch.float64),
            rotation_noise * torch.randn(num_cameras, 3, generator=g, dtype=torch.float64),
        ),
        -1,
    )
    cams0 = cams @ se3_exp(perturb)
    pts0 = pts + point_noise * torch.randn(num_points, 3, generator=g, dtype=torch.float64)
    return BundleAdjustmentData(cams, pts, cams0, pts0, cam_idx, pt_idx, uv)


def small_bundle_adjustment(seed: int = 0) -> BundleAdjustmentData:
    """10 cameras, 500 points, 8 views each: 4,000 observations."""
    return make_bundle_adjustment(10, 500, 8, seed=seed)


def mid_bundle_adjustment(seed: int = 0) -> BundleAdjustmentData:
    """256 cameras, 100,000 points, 10 views within +-60 degrees: 1,000,000 observations."""
    return make_bundle_adjustment(256, 100_000, 10, seed=seed, azimuth_window=math.pi / 3)


def build_bundle_adjustment(data: BundleAdjustmentData, api, *, device="cpu", dtype=torch.float64,
                            loss=None, residual=None):
    """Build a ``Problem`` with camera 0 fixed, using ``api`` (this package or torchls).

    ``residual`` defaults to this package's built-in :func:`reprojection`.
    Group "cams" holds cameras 1..C-1; observations of camera 0 form a second
    residual batch in which the camera is shared constant data.
    """
    if residual is None:
        from .residuals import reprojection as residual
    free, fixed = data.split_fixed_camera()
    problem = api.Problem(
        {
            "cams": data.cameras_init[1:].to(device=device, dtype=dtype),
            "points": data.points_init.to(device=device, dtype=dtype),
        },
        manifolds={"cams": api.SE3Var},
    )
    problem.add_residual(
        residual,
        ("cams", data.camera_index[free] - 1),
        ("points", data.point_index[free]),
        data.uv[free].to(device=device, dtype=dtype),
        loss=loss,
    )
    if bool(fixed.any()):
        problem.add_residual(
            residual,
            data.cameras_true[0].to(device=device, dtype=dtype),
            ("points", data.point_index[fixed]),
            data.uv[fixed].to(device=device, dtype=dtype),
            in_dims=(None, 0, 0),
            loss=loss,
        )
    return problem


def build_differentiable_bundle_adjustment(data: BundleAdjustmentData, api, *, device="cpu", dtype=torch.float64,
                                           loss=None, residual=None):
    """Bundle adjustment with camera 0 fixed, per-observation weights and a
    scale prior (distance of camera 1 from camera 0 at its true value), so
    the solution is an isolated minimum and can be differentiated.

    Returns ``(problem, inputs)``; ``inputs`` holds the observation and weight
    tensors used by the problem ("uv_free", "uv_fixed", "w_free", "w_fixed").
    """
    if residual is None:
        from .residuals import reprojection as residual
    from .residuals import camera_distance_prior

    free, fixed = data.split_fixed_camera()
    problem = api.Problem(
        {
            "cams": data.cameras_init[1:].to(device=device, dtype=dtype),
            "points": data.points_init.to(device=device, dtype=dtype),
        },
        manifolds={"cams": api.SE3Var},
    )
    inputs = {
        "uv_free": data.uv[free].to(device=device, dtype=dtype).clone(),
        "uv_fixed": data.uv[fixed].to(device=device, dtype=dtype).clone(),
        "w_free": torch.ones(int(free.sum()), device=device, dtype=dtype),
        "w_fixed": torch.ones(int(fixed.sum()), device=device, dtype=dtype),
    }
    problem.add_residual(residual, ("cams", data.camera_index[free] - 1), ("points", data.point_index[free]),
                         inputs["uv_free"], loss=loss, weights=inputs["w_free"])
    problem.add_residual(residual, data.cameras_true[0].to(device=device, dtype=dtype),
                         ("points", data.point_index[fixed]), inputs["uv_fixed"], in_dims=(None, 0, 0), loss=loss,
                         weights=inputs["w_fixed"])
    c = lambda T: -(T[:3, :3].T @ T[:3, 3])  # noqa: E731
    dist = torch.linalg.vector_norm(c(data.cameras_true[1]) - c(data.cameras_true[0])).reshape(())
    problem.add_residual(camera_distance_prior, ("cams", torch.tensor([0])),
                         data.cameras_true[0].to(device=device, dtype=dtype), dist.to(device=device, dtype=dtype),
                         in_dims=(0, None, None))
    return problem, inputs


def differentiable_loss(solution, data: BundleAdjustmentData) -> Tensor:
    """Mean squared distance of the solved points to the true points plus the
    squared translation error of the solved (free) camera poses."""
    pts = solution["points"]
    cams = solution["cams"]
    pt = data.points_true.to(pts)
    ct = data.cameras_true[1:].to(cams)
    return ((pts - pt) ** 2).sum(-1).mean() + ((cams[:, :3, 3] - ct[:, :3, 3]) ** 2).sum()


def batched_bundle_adjustment(count: int = 4096, first_seed: int = 0) -> list[BundleAdjustmentData]:
    """Independent problems of uneven size, one per seed: cameras uniform in
    {2..32}, points log-uniform in [20, 2000], each point seen by min(6,
    cameras) distinct cameras (about 2.3M observations for 4,096 problems)."""
    out = []
    for seed in range(first_seed, first_seed + count):
        g = torch.Generator().manual_seed(1_000_003 * seed + 17)
        cams = int(torch.randint(2, 33, (1,), generator=g))
        pts = int(round(math.exp(math.log(20) + (math.log(2000) - math.log(20)) * float(torch.rand(1, generator=g)))))
        out.append(make_bundle_adjustment(cams, pts, min(6, cams), seed=seed))
    return out


@dataclass
class PoseGraphData:
    poses_true: Tensor  # [N, 4, 4]
    poses_init: Tensor  # [N, 4, 4]
    edge_i: Tensor  # [E]
    edge_j: Tensor  # [E]
    measurements: Tensor  # [E, 4, 4]  Z_ij ~ T_i^-1 T_j


def _walk(num_poses, g, yaw_sigma):
    """Unit-step 3D walk: SE(3) poses (yaw only) and positions."""
    yaw = torch.cumsum(yaw_sigma * torch.randn(num_poses, generator=g, dtype=torch.float64), 0)
    pitch = 0.05 * torch.randn(num_poses, generator=g, dtype=torch.float64)
    step = torch.stack((yaw.cos() * pitch.cos(), yaw.sin() * pitch.cos(), pitch.sin()), -1)
    pos = torch.cat((torch.zeros(1, 3, dtype=torch.float64), torch.cumsum(step[:-1], 0)))
    rot_vec = torch.zeros(num_poses, 3, dtype=torch.float64)
    rot_vec[:, 2] = yaw
    poses = se3_exp(torch.cat((torch.zeros_like(rot_vec), rot_vec), -1))
    poses[:, :3, 3] = pos
    return poses, pos


def _loop_candidates(pos, loop_radius):
    """Pose pairs (i, j), j > i + 1, within loop_radius (vectorised in blocks)."""
    cand_i, cand_j = [], []
    block = 2048
    for s in range(0, len(pos), block):
        d = torch.cdist(pos[s : s + block], pos)
        ii, jj = (d <= loop_radius).nonzero(as_tuple=True)
        ii = ii + s
        keep = jj > ii + 1
        cand_i.append(ii[keep])
        cand_j.append(jj[keep])
    return torch.cat(cand_i), torch.cat(cand_j)


def make_sim3_pose_graph(
    num_poses: int = 60,
    num_loops: int = 120,
    *,
    seed: int = 0,
    yaw_sigma: float = 0.3,
    scale_sigma: float = 0.02,
    rotation_noise: float = 0.01,
    translation_noise: float = 0.02,
    scale_noise: float = 0.005,
    loop_radius: float = 3.0,
) -> PoseGraphData:
    from .residuals import sim3_inverse

    g = torch.Generator().manual_seed(seed)
    poses, pos = _walk(num_poses, g, yaw_sigma)
    scale = torch.exp(torch.cumsum(scale_sigma * torch.randn(num_poses, generator=g, dtype=torch.float64), 0))
    poses[:, :3, :3] *= scale[:, None, None]
    cand_i, cand_j = _loop_candidates(pos, loop_radius)
    if cand_i.numel() == 0 and num_loops > 0:
        raise ValueError("no loop-closure candidates")
    pick = torch.randint(cand_i.numel(), (num_loops,), generator=g)
    ei = torch.cat((torch.arange(num_poses - 1), cand_i[pick]))
    ej = torch.cat((torch.arange(1, num_poses), cand_j[pick]))
    rel = sim3_inverse(poses[ei]) @ poses[ej]
    noise = torch.cat(
        (
            translation_noise * torch.randn(len(ei), 3, generator=g, dtype=torch.float64),
            rotation_noise * torch.randn(len(ei), 3, generator=g, dtype=torch.float64),
            scale_noise * torch.randn(len(ei), 1, generator=g, dtype=torch.float64),
        ),
        -1,
    )
    meas = rel @ sim3_exp(noise)
    init = [poses[0]]
    for k in range(num_poses - 1):
        init.append(init[-1] @ meas[k])
    return PoseGraphData(poses, torch.stack(init), ei, ej, meas)


def make_pose_graph(
    num_poses: int = 1000,
    num_loops: int = 3000,
    *,
    seed: int = 0,
    yaw_sigma: float = 0.1,
    rotation_noise: float = 0.01,
    translation_noise: float = 0.02,
    loop_radius: float = 3.0,
) -> PoseGraphData:
    g = torch.Generator().manual_seed(seed)
    poses, pos = _walk(num_poses, g, yaw_sigma)
    cand_i, cand_j = _loop_candidates(pos, loop_radius)
    if cand_i.numel() == 0 and num_loops > 0:
        raise ValueError("no loop-closure candidates")
    pick = torch.randint(cand_i.numel(), (num_loops,), generator=g)
    ei = torch.cat((torch.arange(num_poses - 1), cand_i[pick]))
    ej = torch.cat((torch.arange(1, num_poses), cand_j[pick]))
    rel = se3_inverse(poses[ei]) @ poses[ej]
    noise = torch.cat(
        (
            translation_noise * torch.randn(len(ei), 3, generator=g, dtype=torch.float64),
            rotation_noise * torch.randn(len(ei), 3, generator=g, dtype=torch.float64),
        ),
        -1,
    )
    meas = rel @ se3_exp(noise)
    init = [poses[0]]
    for k in range(num_poses - 1):
        init.append(init[-1] @ meas[k])
    return PoseGraphData(poses, torch.stack(init), ei, ej, meas)


def build_pose_graph(data: PoseGraphData, api, *, device="cpu", dtype=torch.float64, loss=None,
                     residual=None, sim3=False):
    """``Problem`` over poses 1..N-1; pose 0 is constant data in its edges.
    ``sim3``: Sim(3) poses with the ``sim3_between`` residual."""
    if residual is None:
        if sim3:
            from .residuals import sim3_between as residual
        else:
            from .residuals import se3_between as residual
    problem = api.Problem(
        {"poses": data.poses_init[1:].to(device=device, dtype=dtype)},
        manifolds={"poses": api.Sim3Var if sim3 else api.SE3Var},
    )
    free = (data.edge_i > 0) & (data.edge_j > 0)
    problem.add_residual(
        residual,
        ("poses", data.edge_i[free] - 1),
        ("poses", data.edge_j[free] - 1),
        data.measurements[free].to(device=device, dtype=dtype),
        loss=loss,
    )
    first = data.edge_i == 0
    if bool(first.any()):
        problem.add_residual(
            residual,
            data.poses_true[0].to(device=device, dtype=dtype),
            ("poses", data.edge_j[first] - 1),
            data.measurements[first].to(device=device, dtype=dtype),
            in_dims=(None, 0, 0),
            loss=loss,
        )
    return problem
