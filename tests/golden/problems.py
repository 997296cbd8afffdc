"""Seeded parity problems shared by the golden-fixture script, the tests and smoke().

Every builder takes ``api`` -- this package, torchls itself, or the oracle
adapter -- and returns a ``Problem`` built through that API's
``Problem.add_residual`` with identical arrays, plus the solve options the
fixture records.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from torchls_b200 import synthetic
from torchls_b200.residuals import reprojection, se3_between


# ---------------------------------------------------------------- residuals used by fixtures
def point_prior(point, reference):
    return point - reference


def curve_residual(params, x, y):
    """Exponential decay fit a * exp(-b x) + c - y (Euclidean, bounded)."""
    return (params[0] * torch.exp(-params[1] * x) + params[2] - y).reshape(1)


def rotation_error(rot_i, rot_j, measured):
    from torchls_b200.geometry import so3_log

    return so3_log(rot_j @ rot_i.T @ measured.T)


def alias_residual(a, b, target):
    """Two slots that may reference the same variable (aliasing)."""
    return torch.stack((a[0] * b[1] - target[0], a[1] + 2 * b[0] - target[1], a[0] - b[0]))


def cam_point_link(cam_offset, point, target):
    """Joint-group residual: a Euclidean camera offset and a point."""
    return cam_offset + point - target


def cauchy_loss(api, scale=0.05):
    """rho(s) = c^2 log(1 + s/c^2); rho'' < 0, so the curvature correction is skipped."""

    class CauchyLoss(api.Loss):
        def evaluate(self, s):
            c2 = scale**2
            return c2 * torch.log1p(s / c2), 1 / (1 + s / c2), -1 / (c2 * (1 + s / c2) ** 2)

    return CauchyLoss()


def soft_square_loss(api):
    """rho(s) = s + s^2/4: rho'' > 0 exercises the full Triggs correction."""

    class SoftSquareLoss(api.Loss):
        def evaluate(self, s):
            return s + 0.25 * s * s, 1 + 0.5 * s, 0.5 + 0 * s

    return SoftSquareLoss()


def se2_between(a, b, z):
    """SE(2) relative-pose error: b expressed in a's frame minus z, angle wrapped."""
    c, s = torch.cos(a[2]), torch.sin(a[2])
    dx, dy = b[0] - a[0], b[1] - a[1]
    e = torch.stack((c * dx + s * dy - z[0], -s * dx + c * dy - z[1], b[2] - a[2] - z[2]))
    return torch.stack((e[0], e[1], torch.atan2(torch.sin(e[2]), torch.cos(e[2]))))


def se2_odometry(a, b, k, z):
    """Odometry edge whose measured translation is in units of an unknown scale k."""
    return se2_between(a, b, torch.stack((k[0] * z[0], k[0] * z[1], z[2])))


def focal_reprojection(camera, focal, point, observation):
    """Reprojection with a per-camera focal scale (a second retained group that
    shares residuals with the camera poses)."""
    xyz = camera[:3, :3] @ point + camera[:3, 3]
    valid = xyz[2] > 1e-6
    z = torch.where(valid, xyz[2], torch.ones_like(xyz[2]))
    err = focal[0] * xyz[:2] / z - observation
    return torch.where(valid, err, torch.zeros_like(err))


def camera_link(cam_a, cam_b, target):
    """Relative position prior between two cameras' translations (couples them)."""
    return cam_a[:3, 3] - cam_b[:3, 3] - target


# ---------------------------------------------------------------- builders
def ba_small(api, device="cpu", dtype=torch.float64, data=None):
    data = data if data is not None else synthetic.small_bundle_adjustment(0)
    return synthetic.build_bundle_adjustment(data, api, device=device, dtype=dtype, loss=api.HuberLoss(0.01))


def ba_tiny(api, device="cpu", dtype=torch.float64, loss=True):
    """4 cameras, 40 points, 3 views: 120 observations (fast per-kernel parity)."""
    data = synthetic.make_bundle_adjustment(4, 40, 3, seed=7)
    return synthetic.build_bundle_adjustment(
        data, api, device=device, dtype=dtype, loss=api.HuberLoss(0.01) if loss else None)


def pose_small(api, device="cpu", dtype=torch.float64):
    data = synthetic.make_pose_graph(80, 300, seed=3, yaw_sigma=0.5)
    return synthetic.build_pose_graph(data, api, device=device, dtype=dtype)


def sim3_small(api, device="cpu", dtype=torch.float64):
    """Sim(3) pose graph: 20 poses, 19 odometry + 60 loop edges (sim3_between)."""
    data = synthetic.make_sim3_pose_graph(20, 60, seed=5)
    return synthetic.build_pose_graph(data, api, device=device, dtype=dtype, sim3=True)


def se2_custom(api, device="cpu", dtype=torch.float64):
    """SE(2) pose graph (``SE2Var``) plus an unknown odometry scale held by a
    user manifold (``PositiveVar``: a positive scalar updated as x * exp(delta),
    no CUDA kind, so its retraction runs through torch on the device):
    16 poses, 15 scaled odometry edges and 24 loop edges; pose 0 is data."""

    class PositiveVar(api.Var, default_factory=lambda: torch.ones(1), tangent_dim=1,
                      retract_fn=lambda x, d: x * torch.exp(d)):
        """Positive scalar, multiplicative update."""

    g = torch.Generator().manual_seed(23)
    n, loops, scale = 16, 24, 1.3
    th = torch.cumsum(0.3 * torch.randn(n, generator=g, dtype=torch.float64), 0)
    xy = torch.cat((torch.zeros(1, 2, dtype=torch.float64),
                    torch.cumsum(torch.stack((th.cos(), th.sin()), -1)[:-1], 0)))
    truth = torch.cat((xy, th[:, None]), -1)

    def rel(i, j):
        return torch.stack([se2_between(truth[a], truth[b], torch.zeros(3, dtype=torch.float64)) for a, b in zip(i, j)])

    oi, oj = torch.arange(n - 1), torch.arange(1, n)
    odo = rel(oi, oj) + 0.01 * torch.randn(n - 1, 3, generator=g, dtype=torch.float64)
    odo[:, :2] /= scale
    li = torch.randint(1, n - 2, (loops,), generator=g)
    lj = torch.minimum(li + torch.randint(2, 6, (loops,), generator=g), torch.tensor(n - 1))
    loop = rel(li, lj) + 0.01 * torch.randn(loops, 3, generator=g, dtype=torch.float64)
    init = [truth[0]]
    for k in range(n - 1):  # integrate odometry at unit scale
        c, s_ = torch.cos(init[-1][2]), torch.sin(init[-1][2])
        z = odo[k]
        init.append(torch.stack((init[-1][0] + c * z[0] - s_ * z[1], init[-1][1] + s_ * z[0] + c * z[1],
                                 init[-1][2] + z[2])))
    to = dict(device=device, dtype=dtype)
    p = api.Problem({"poses": torch.stack(init[1:]).to(**to), "scale": torch.ones(1, 1, **to)},
                    manifolds={"poses": api.SE2Var, "scale": PositiveVar})
    zero = lambda m: torch.zeros(m, dtype=torch.long)  # noqa: E731
    p.add_residual(se2_odometry, ("poses", oi[1:] - 1), ("poses", oj[1:] - 1), ("scale", zero(n - 2)),
                   odo[1:].to(**to))
    p.add_residual(se2_odometry, truth[0].to(**to), ("poses", torch.tensor([0])), ("scale", zero(1)),
                   odo[:1].to(**to), in_dims=(None, 0, 0, 0))
    p.add_residual(se2_between, ("poses", li - 1), ("poses", lj - 1), loop.to(**to))
    return p


def _tiny_data():
    return synthetic.make_bundle_adjustment(4, 40, 3, seed=7)


def ba_two_groups(api, device="cpu", dtype=torch.float64):
    """The tiny BA with its free cameras split into two retained groups
    ("cams_a": cameras 1-2, "cams_b": camera 3); no residual couples them."""
    d = _tiny_data()
    to = dict(device=device, dtype=dtype)
    p = api.Problem({"cams_a": d.cameras_init[1:3].to(**to), "cams_b": d.cameras_init[3:4].to(**to),
                     "points": d.points_init.to(**to)}, manifolds={"cams_a": api.SE3Var, "cams_b": api.SE3Var})
    huber = api.HuberLoss(0.01)
    for name, sel, base in (("cams_a", (d.camera_index >= 1) & (d.camera_index <= 2), 1),
                            ("cams_b", d.camera_index == 3, 3)):
        p.add_residual(reprojection, (name, d.camera_index[sel] - base), ("points", d.point_index[sel]),
                       d.uv[sel].to(**to), loss=huber)
    fixed = d.camera_index == 0
    p.add_residual(reprojection, d.cameras_true[0].to(**to), ("points", d.point_index[fixed]), d.uv[fixed].to(**to),
                   in_dims=(None, 0, 0), loss=huber)
    return p


def ba_priors(api, device="cpu", dtype=torch.float64):
    """The tiny BA plus relative-position priors between consecutive free
    cameras: residuals that couple two retained variables."""
    p = ba_tiny(api, device=device, dtype=dtype)
    d = _tiny_data()
    a, b = torch.tensor([0, 1]), torch.tensor([1, 2])
    target = (d.cameras_true[1 + a, :3, 3] - d.cameras_true[1 + b, :3, 3]).to(device=device, dtype=dtype)
    p.add_residual(camera_link, ("cams", a), ("cams", b), target,
                   weights=torch.full((2,), 0.5, dtype=dtype, device=device))
    return p


def ba_intrinsics(api, device="cpu", dtype=torch.float64):
    """The tiny BA with a per-camera focal scale ("focal", 1-dim, cameras 1-3)
    entering the reprojection of the free cameras (two retained groups coupled
    in every residual) and a weak prior holding each focal near 1."""
    d = _tiny_data()
    to = dict(device=device, dtype=dtype)
    true_f = torch.tensor([1.0, 1.05, 0.97, 1.02], dtype=torch.float64)
    uv = d.uv * true_f[d.camera_index][:, None]
    p = api.Problem({"cams": d.cameras_init[1:].to(**to), "focal": torch.ones(3, 1, **to),
                     "points": d.points_init.to(**to)}, manifolds={"cams": api.SE3Var})
    huber = api.HuberLoss(0.01)
    free = d.camera_index > 0
    p.add_residual(focal_reprojection, ("cams", d.camera_index[free] - 1), ("focal", d.camera_index[free] - 1),
                   ("points", d.point_index[free]), uv[free].to(**to), loss=huber)
    p.add_residual(reprojection, d.cameras_true[0].to(**to), ("points", d.point_index[~free]), uv[~free].to(**to),
                   in_dims=(None, 0, 0), loss=huber)
    p.add_residual(point_prior, ("focal", torch.arange(3)), torch.ones(3, 1, **to),
                   weights=torch.full((3,), 1e-2, dtype=dtype, device=device))
    return p


def typed_ba(api, device="cpu", dtype=torch.float64):
    """The tiny bundle adjustment through the typed API (``Cost.factory``,
    ``Cost``, ``LeastSquaresProblem``, ``VarValues.make``) with sparse, unsorted
    IDs: free cameras 30, 10, 20 (camera 0 is constant data), points
    100 + 3 * (39 - p). Returns the analysed problem and the initial values."""
    data = synthetic.make_bundle_adjustment(4, 40, 3, seed=7)

    class PointVar(api.Var, default_factory=lambda: torch.zeros(3)):
        """A Euclidean 3-vector (typed API)."""

    cam_ids = torch.tensor([30, 10, 20])
    pt_ids = 100 + 3 * torch.arange(39, -1, -1)
    free, fixed = data.split_fixed_camera()
    to = dict(device=device, dtype=dtype)
    huber = api.HuberLoss(0.01)
    observe = api.Cost.factory(reprojection, loss=huber)
    costs = [
        observe(api.SE3Var(cam_ids[data.camera_index[free] - 1]), PointVar(pt_ids[data.point_index[free]]),
                data.uv[free].to(**to)),
        api.Cost(reprojection, (data.cameras_true[0].to(**to), PointVar(pt_ids[data.point_index[fixed]]),
                                data.uv[fixed].to(**to)), in_dims=(None, 0, 0), loss=huber),
    ]
    problem = api.LeastSquaresProblem(costs, [PointVar(pt_ids), api.SE3Var(cam_ids)]).analyze()
    init = api.VarValues.make([api.SE3Var(cam_ids).with_value(data.cameras_init[1:].to(**to)),
                               PointVar(pt_ids).with_value(data.points_init.to(**to))])
    return problem, init


def sim3_exp_cases():
    """Seeded Sim(3) poses and tangents [t, w, log s] for known-answer tests of
    the retraction X * Exp(delta): zero, tiny, small and moderate tangents,
    rotations near pi and large scale changes."""
    from torchls_b200.geometry import sim3_exp

    g = torch.Generator().manual_seed(29)
    rnd = lambda n, s: s * torch.randn(n, 7, generator=g, dtype=torch.float64)
    axis = torch.nn.functional.normalize(torch.randn(4, 3, generator=g, dtype=torch.float64), dim=-1)
    near_pi = torch.cat((rnd(4, 0.5)[:, :3], axis * 3.1, torch.tensor([[0.3], [-0.2], [0.0], [1e-9]],
                                                                        dtype=torch.float64)), -1)
    big_scale = rnd(4, 0.01)
    big_scale[:, 6] = torch.tensor([1.5, -1.5, 2.5, -2.5], dtype=torch.float64)
    delta = torch.cat((torch.zeros(1, 7, dtype=torch.float64), rnd(3, 1e-9), rnd(3, 1e-5), rnd(3, 1e-2),
                       rnd(4, 0.5), near_pi, big_scale, rnd(4, 1.0)))
    pose = sim3_exp(rnd(len(delta), 0.7))
    return pose, delta


def curve_bounds(api, device="cpu", dtype=torch.float64):
    g = torch.Generator().manual_seed(5)
    x = torch.linspace(0, 4, 60, dtype=torch.float64)
    y = 2.0 * torch.exp(-1.3 * x) + 0.5 + 0.01 * torch.randn(60, generator=g, dtype=torch.float64)
    p = api.Problem({"params": torch.tensor([[1.0, 0.5, 0.7]], dtype=dtype, device=device)})
    p.add_residual(curve_residual, ("params", torch.zeros(60, dtype=torch.long)),
                   x.to(device=device, dtype=dtype), y.to(device=device, dtype=dtype))
    return p


CURVE_BOUNDS = {"params": ([0.0, 0.0, 0.6], [1.8, 5.0, 1.0])}


def rotations_small(api, device="cpu", dtype=torch.float64):
    from torchls_b200.geometry import so3_exp

    g = torch.Generator().manual_seed(11)
    n = 12
    truth = so3_exp(0.4 * torch.randn(n, 3, generator=g, dtype=torch.float64))
    ii, jj = torch.triu_indices(n, n, offset=1)
    noise = so3_exp(0.01 * torch.randn(len(ii), 3, generator=g, dtype=torch.float64))
    rel = noise @ truth[jj] @ truth[ii].transpose(-1, -2)
    init = truth @ so3_exp(0.1 * torch.randn(n, 3, generator=g, dtype=torch.float64))
    p = api.Problem({"rot": init[1:].to(device=device, dtype=dtype)}, manifolds={"rot": api.SO3Var})
    free = (ii > 0)
    p.add_residual(rotation_error, ("rot", ii[free] - 1), ("rot", jj[free] - 1),
                   rel[free].to(device=device, dtype=dtype), loss=api.HuberLoss(math.radians(2)))
    p.add_residual(rotation_error, truth[0].to(device=device, dtype=dtype), ("rot", jj[~free] - 1),
                   rel[~free].to(device=device, dtype=dtype), in_dims=(None, 0, 0))
    return p


def alias_weights(api, device="cpu", dtype=torch.float64, loss=None):
    g = torch.Generator().manual_seed(13)
    m = 30
    vals = torch.randn(6, 2, generator=g, dtype=torch.float64)
    a = torch.randint(0, 6, (m,), generator=g)
    b = torch.randint(0, 6, (m,), generator=g)
    b[:8] = a[:8]  # aliased slots
    tgt = torch.randn(m, 3, generator=g, dtype=torch.float64)
    w = torch.rand(m, generator=g, dtype=torch.float64) + 0.5
    p = api.Problem({"v": vals.to(device=device, dtype=dtype)})
    p.add_residual(alias_residual, ("v", a), ("v", b), tgt[:, :2].to(device=device, dtype=dtype),
                   weights=w.to(device=device, dtype=dtype), loss=loss)
    p.add_residual(point_prior, ("v", torch.arange(6)), torch.zeros(6, 2, dtype=dtype, device=device))
    return p


def joint_groups(api, device="cpu", dtype=torch.float64):
    """Two Euclidean groups with identical IDs, coupled per observation."""
    g = torch.Generator().manual_seed(17)
    n, m = 8, 40
    off0 = 0.1 * torch.randn(n, 3, generator=g, dtype=torch.float64)
    pts0 = torch.randn(n, 3, generator=g, dtype=torch.float64)
    idx = torch.randint(0, n, (m,), generator=g)
    tgt = torch.randn(m, 3, generator=g, dtype=torch.float64)
    p = api.Problem({"off": off0.to(device=device, dtype=dtype), "pts": pts0.to(device=device, dtype=dtype)})
    p.add_residual(cam_point_link, ("off", idx), ("pts", idx), tgt.to(device=device, dtype=dtype))
    p.add_residual(point_prior, ("off", torch.arange(n)), torch.zeros(n, 3, dtype=dtype, device=device))
    p.add_residual(point_prior, ("pts", torch.arange(n)), torch.zeros(n, 3, dtype=dtype, device=device))
    return p


# ---------------------------------------------------------------- oracle adapter
class OracleAPI:
    """Exposes the oracle through the same Problem / Var / loss names."""

    SE3Var = "se3"
    SO3Var = "so3"
    Sim3Var = "sim3"
    Loss = object

    @staticmethod
    def HuberLoss(delta):
        from oracle.model import huber_loss

        return huber_loss(delta)

    class Problem:
        def __init__(self, parameters, manifolds=None):
            from oracle.model import OracleProblem

            params = {k: np.asarray(v.detach().cpu().numpy(), dtype=np.float64) for k, v in parameters.items()}
            self.inner = OracleProblem(params, dict(manifolds or {}))

        def add_residual(self, fn, *args, in_dims=None, loss=None, weights=None, **_):
            from oracle.model import generic_loss, huber_loss

            conv = []
            for a in args:
                if isinstance(a, tuple):
                    conv.append((a[0], np.asarray(torch.as_tensor(a[1]).cpu().numpy())))
                else:
                    conv.append(np.asarray(torch.as_tensor(a).detach().cpu().numpy()))
            if loss is not None and not isinstance(loss, huber_loss):
                inner_loss = loss

                def ev(s):
                    out = inner_loss.evaluate(torch.as_tensor(s))
                    return tuple(np.broadcast_to(np.asarray(o, dtype=np.float64), s.shape) for o in out)

                loss = generic_loss(ev)
            w = None if weights is None else np.asarray(torch.as_tensor(weights).cpu().numpy())
            self.inner.add_residual(fn, *conv, in_dims=in_dims, loss=loss, weights=w)
            return self


def oracle_problem(builder, **kw):
    return builder(OracleAPI, **kw).inner


def fixed_system_case():
    """A seeded sparse 240 x 30 matrix (about 4 entries per row), two
    right-hand sides, row weights and an LAD target with 10 % gross outliers."""
    g = torch.Generator().manual_seed(41)
    m, n = 240, 30
    A = torch.zeros(m, n, dtype=torch.float64)
    for r in range(m):
        cols = torch.randperm(n, generator=g)[:4]
        A[r, cols] = torch.randn(4, generator=g, dtype=torch.float64)
    x = torch.randn(n, 2, generator=g, dtype=torch.float64)
    y = torch.randn(m, 2, generator=g, dtype=torch.float64)
    w = torch.rand(m, generator=g, dtype=torch.float64) + 0.2
    truth = torch.randn(n, 2, generator=g, dtype=torch.float64)
    target = A @ truth + 0.01 * torch.randn(m, 2, generator=g, dtype=torch.float64)
    bad = torch.randperm(m, generator=g)[: m // 10]
    target[bad] += 5.0 * torch.randn(len(bad), 2, generator=g, dtype=torch.float64)
    return A, x, y, w, target
