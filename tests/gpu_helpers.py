"""Shared helpers for the GPU parity tests."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest
import torch

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SUMMARIES = json.load(open(os.path.join(HERE, "summaries.json")))

needs_gpu = pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")


def load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


def stored_ba(fx):
    from torchls_b200.synthetic import BundleAdjustmentData

    keys = ("cameras_true", "points_true", "cameras_init", "points_init", "camera_index", "point_index", "uv")
    return BundleAdjustmentData(**{k: torch.from_numpy(fx[k]) for k in keys})


def to_np(x):
    return x.detach().cpu().numpy() if torch.is_tensor(x) else np.asarray(x)


def close(a, b, rtol, atol=0.0, what=""):
    a, b = np.asarray(to_np(a), dtype=np.float64), np.asarray(to_np(b), dtype=np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    scale = max(np.abs(b).max(initial=0.0), 1e-300)
    err = np.abs(a - b).max(initial=0.0)
    assert err <= rtol * scale + atol, f"{what}: max err {err:.3e} vs scale {scale:.3e} (rtol {rtol:g})"


def check_summary(s, ref, *, histories=True, counts=True, cost_rtol=1e-10, cg_slack=0):
    """Compare a SolveSummary with the reference's.

    ``cg_slack`` allows CG iteration counts to differ by that many per linear
    solve: for CG runs of ~180 iterations the float64 summation order of the
    dot products (deterministic but not torch's) can move the rtol crossing
    by one iteration.
    """
    assert s.termination_reason == ref["termination_reason"], (s.termination_reason, ref["termination_reason"])
    close(s.final_cost, ref["final_cost"], cost_rtol, what="final_cost")
    if not counts:
        return
    assert s.iterations == ref["iterations"]
    assert s.accepted_steps == ref["accepted_steps"]
    assert s.rejected_steps == ref["rejected_steps"]
    close(s.initial_cost, ref["initial_cost"], 1e-12, what="initial_cost")
    if histories:
        got, want = s.linear_iterations_history, ref["linear_iterations_history"]
        assert len(got) == len(want) and all(abs(a - b) <= cg_slack for a, b in zip(got, want)), (got, want)
        close(s.lambda_history, ref["lambda_history"], 1e-12, what="lambda_history")
        close(s.cost_history, ref["cost_history"], 1e-8, what="cost_history")
