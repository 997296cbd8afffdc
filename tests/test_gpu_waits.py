"""Bounded device waits of the persistent Schur-PCG kernels.

Every wait in the Schur kernels (a bulk copy landing in shared memory, a grid
barrier, the vector CTA's arrivals) gives up after ``SchurPlan.wait_cycles``
SM cycles, sets the plan's device error word and lets every CTA leave. Here the
limit is cut to 200 cycles on the small bundle adjustment: the CTAs that have
no chunks reach the first grid barrier microseconds before the CTAs streaming
chunks, so their waits run out on every launch. The solve must return to the
host and raise ``RuntimeError``; with the default limit restored, the same
cached plan must solve again to the same result (the error word is cleared per
damped system). No wait is unbounded, and a CTA whose bulk-copy wait runs out
reads nothing from that stage, so a cut limit never leads to an out-of-bounds
access: it only gives wrong numbers that the error word marks.
"""

from __future__ import annotations

import pytest
import torch

from gpu_helpers import close, load, needs_gpu, stored_ba
from golden import problems as P

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _solve(tls, prob, start):
    # a solve writes its result back into the problem: start each from the same values
    prob.parameters.update({k: v.clone() for k, v in start.items()})
    return prob.solve(return_summary=True, linear_solver="schur_cg", eliminate="points",
                      termination=tls.TerminationConfig(max_iterations=30))


def test_expired_wait_raises_and_plan_recovers():
    import torchls_b200 as tls

    fx = load("ba_small")
    prob = P.ba_small(tls, device=DEV, data=stored_ba(fx))
    start = {k: v.clone() for k, v in prob.parameters.items()}
    sol0, s0 = _solve(tls, prob, start)
    assert s0.linear_iterations > 0
    plans = list(prob._ensure_analyzed().__dict__["_schur_plans"].values())
    assert len(plans) == 1
    plan = plans[0]
    plan.wait_cycles = 200
    with pytest.raises(RuntimeError, match="bounded device wait"):
        _solve(tls, prob, start)
    torch.cuda.synchronize()
    assert int(plan.err.item()) != 0  # the kernel returned with its error word set
    plan.wait_cycles = 0
    sol1, s1 = _solve(tls, prob, start)
    assert int(plan.err.item()) == 0
    assert s1.linear_iterations_history == s0.linear_iterations_history
    close(s1.final_cost, s0.final_cost, 1e-14, what="final cost after recovery")
    close(sol1["cams"], sol0["cams"], 1e-12, what="cams after recovery")
