"""Batched solve of independent problems (per-problem damping and masks).

Every problem of a batch must reach the cost its own solve reaches (same
generator, same LM settings): the gauge of each bundle adjustment (global
scale with camera 0 fixed) leaves the parameters free along a line, so the
comparison is on final costs, to 1e-6 relative.
"""

from __future__ import annotations

import pytest
import torch

from gpu_helpers import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def test_batched_matches_individual_solves():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.batched import solve_batched

    datas = synthetic.batched_bundle_adjustment(10, first_seed=100)
    build = lambda d: synthetic.build_bundle_adjustment(d, tls, device=DEV, loss=tls.HuberLoss(0.01))  # noqa: E731
    sols, summary = solve_batched([build(d) for d in datas], max_iterations=30)
    assert summary.problems == 10
    for j, d in enumerate(datas):
        prob = build(d)
        _, s = prob.solve(return_summary=True, linear_solver="schur_cg", eliminate="points",
                          termination=tls.TerminationConfig(max_iterations=30))
        got = float(summary.final_cost[j])
        assert abs(got - s.final_cost) <= 1e-6 * s.final_cost + 1e-14, (j, got, s.final_cost,
                                                                          summary.termination[j])
        assert summary.termination[j] in ("gradient_tolerance", "cost_tolerance"), summary.termination[j]
        # the returned solution evaluates to the reported cost
        cost = float(prob.cost(sols[j]))
        assert abs(cost - got) <= 1e-9 * got


def test_batched_single_problem_and_inactive_blocks():
    import torchls_b200 as tls
    from torchls_b200 import synthetic
    from torchls_b200.batched import solve_batched

    d = synthetic.make_bundle_adjustment(4, 40, 3, seed=7)
    prob = synthetic.build_bundle_adjustment(d, tls, device=DEV, loss=tls.HuberLoss(0.01))
    init = {k: v.clone() for k, v in prob.parameters.items()}
    sols, summary = solve_batched([prob], max_iterations=30)
    prob.parameters = init
    _, s = prob.solve(return_summary=True, linear_solver="schur_cg", eliminate="points",
                      termination=tls.TerminationConfig(max_iterations=30))
    assert abs(float(summary.final_cost[0]) - s.final_cost) <= 1e-6 * s.final_cost
    assert torch.isfinite(sols[0]["cams"]).all()


@pytest.mark.parametrize("precision", ["native", "mixed"])
def test_batched_matches_oracle(precision):
    """Batched final costs against the numpy oracle (the reference's float64
    LM with Schur-PCG, solved problem by problem on the host) on four problems
    of the batched generator, in float64 and in mixed precision (float32 J and
    W storage): 1e-6 relative, the tolerance of the batched-vs-individual test."""
    import oracle
    import torchls_b200 as tls
    from golden import problems as P
    from torchls_b200 import synthetic
    from torchls_b200.batched import solve_batched

    datas = synthetic.batched_bundle_adjustment(4, first_seed=200)
    build = lambda d, api, **k: synthetic.build_bundle_adjustment(d, api, loss=api.HuberLoss(0.01), **k)  # noqa: E731
    _, summary = solve_batched([build(d, tls, device=DEV) for d in datas], max_iterations=30, precision=precision)
    for j, d in enumerate(datas):
        _, ref = oracle.solve(P.oracle_problem(lambda api, d=d: build(d, api)), linear_solver="schur_cg",
                              eliminate="points", termination=dict(max_iterations=30))
        got = float(summary.final_cost[j])
        assert abs(got - ref.final_cost) <= 1e-6 * ref.final_cost + 1e-14, (j, got, ref.final_cost)
