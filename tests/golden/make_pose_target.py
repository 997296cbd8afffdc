"""Reference float64 solve of the SE(3) pose graph (100,000 poses, 399,999 edges).

    python tests/golden/make_pose_target.py /path/to/torchls-checkout [--poses N --loops M]

Runs torchls itself on CPU (float64): full-system conjugate-gradient LM with
block-Jacobi on the 6x6 pose blocks, 30 LM iterations, on the seeded
generator of ``torchls_b200.synthetic.make_pose_graph`` (unit steps, yaw
increments N(0, 0.1^2), 300,000 loop closures drawn with replacement among
pose pairs within 3 m, noise N(0, 0.01^2) rad and N(0, 0.02^2) m, initial
values composed from the noisy odometry, pose 0 held fixed as constant data).
The residual is log(Z^-1 T_i^-1 T_j) from ``torchls_b200.residuals.se3_between``
(plain torch ops; the reference ships no SE(3) logarithm). Writes
``tests/golden/pose_graph_target.json`` with the final cost and histories
(``--poses 10000 --loops 30000``: the same generator at a tenth of the size,
where CG still stops at its 200-iteration cap every LM iteration, written to
``pose_graph_10k_target.json``).
"""

from __future__ import annotations

import json
import os
import sys
import time

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

POSES, LOOPS, SEED, ITERATIONS = 100_000, 300_000, 0, 30


def main(reference, poses=POSES, loops=LOOPS):
    sys.path.insert(0, reference)
    import torchls as tls

    from torchls_b200 import synthetic
    from torchls_b200.residuals import se3_between

    torch.set_num_threads(os.cpu_count())
    t0 = time.perf_counter()
    data = synthetic.make_pose_graph(poses, loops, seed=SEED)
    gen_s = time.perf_counter() - t0
    prob = synthetic.build_pose_graph(data, tls, residual=se3_between)
    t0 = time.perf_counter()
    _, s = prob.solve(return_summary=True, linear_solver="conjugate_gradient",
                      termination=tls.TerminationConfig(max_iterations=ITERATIONS))
    seconds = time.perf_counter() - t0
    out = dict(final_cost=s.final_cost, initial_cost=s.initial_cost, iterations=s.iterations,
               termination_reason=s.termination_reason, cost_history=s.cost_history,
               lambda_history=s.lambda_history, linear_iterations_history=s.linear_iterations_history,
               cpu_seconds_cold=seconds, cpu_threads=torch.get_num_threads(), generator_seconds=gen_s,
               poses=poses, edges=int(data.edge_i.numel()),
               linear_relative_residual_history=s.linear_relative_residual_history)
    name = "pose_graph_target.json" if poses == POSES else f"pose_graph_{poses // 1000}k_target.json"
    with open(os.path.join(HERE, name), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else os.environ.get(
        "TORCHLS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the torchls checkout> "
                 "(or set TORCHLS_REFERENCE)")
    arg = lambda flag, default: int(sys.argv[sys.argv.index(flag) + 1]) if flag in sys.argv else default  # noqa: E731
    main(ref, arg("--poses", POSES), arg("--loops", LOOPS))
