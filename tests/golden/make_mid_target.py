"""Reference float64 solve of the mid-size bundle adjustment (1,000,000 observations).

    python tests/golden/make_mid_target.py /path/to/torchls-checkout

Runs torchls itself on CPU (float64) with the benchmark's settings and writes
``tests/golden/ba_mid_target.json``: the final cost the GPU solves must reach
within 1e-8 relative, plus the reference's LM/CG histories and timing.
"""

from __future__ import annotations

import json
import os
import sys
import time

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(reference):
    sys.path.insert(0, reference)
    import torchls as tls

    from torchls_b200 import synthetic

    torch.set_num_threads(os.cpu_count())
    data = synthetic.mid_bundle_adjustment(0)
    prob = synthetic.build_bundle_adjustment(data, tls, loss=tls.HuberLoss(0.01))
    t0 = time.perf_counter()
    _, s = prob.solve(return_summary=True, linear_solver="schur_cg", eliminate="points",
                      termination=tls.TerminationConfig(max_iterations=20))
    seconds = time.perf_counter() - t0
    out = dict(final_cost=s.final_cost, initial_cost=s.initial_cost, iterations=s.iterations,
               termination_reason=s.termination_reason, cost_history=s.cost_history,
               lambda_history=s.lambda_history, linear_iterations_history=s.linear_iterations_history,
               cpu_seconds_cold=seconds, cpu_threads=torch.get_num_threads(),
               observations=data.num_observations)
    with open(os.path.join(HERE, "ba_mid_target.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCHLS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the torchls checkout> "
                 "(or set TORCHLS_REFERENCE)")
    main(ref)
