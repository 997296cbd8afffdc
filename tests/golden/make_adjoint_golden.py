"""Golden gradients of a bundle-adjustment solution from the reference's own
float64 Gauss-Newton steps, differentiated by torch.autograd.

    python tests/golden/make_adjoint_golden.py /path/to/torchls-checkout

Problem: the 10-camera / 500-point / 4,000-observation bundle adjustment
(seed 0) with camera 0 fixed, Huber 0.01 and a prior on the distance of
camera 1 from camera 0 (removes the scale gauge). torchls builds the problem
(its linearization is connected to the observation tensors); the script
unrolls K Gauss-Newton steps through ``AnalyzedLeastSquaresProblem.linearize``,
``BlockJacobian.to_dense``, a dense solve and ``_NamedValues.retract``, and
differentiates the loss (mean squared distance of the solved points to the
true points plus the squared translation error of the free cameras) with
respect to every observation. Two unroll lengths are compared to show the
derivative has converged. Writes ``tests/golden/adjoint_small.npz``.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def unrolled(tls, steps):
    from torchls_b200 import synthetic

    data = synthetic.small_bundle_adjustment(0)
    prob, inputs = synthetic.build_differentiable_bundle_adjustment(data, tls, loss=tls.HuberLoss(0.01))
    uv = [inputs["uv_free"].requires_grad_(True), inputs["uv_fixed"].requires_grad_(True)]
    an, vals = prob._state(None)
    for _ in range(steps):
        lin = an.linearize(vals)
        J = lin.jacobian.to_dense()
        r = lin.residual
        delta = -torch.linalg.solve(J.T @ J, J.T @ r)
        vals = vals.retract(delta, an.layout)
    sol = dict(vals._values)
    loss = synthetic.differentiable_loss(sol, data)
    grads = torch.autograd.grad(loss, uv)
    return loss.detach(), [g.detach() for g in grads], {k: v.detach() for k, v in sol.items()}


def main(reference):
    sys.path.insert(0, reference)
    import torchls as tls

    torch.set_num_threads(os.cpu_count())
    loss_a, ga, sol_a = unrolled(tls, 12)
    loss_b, gb, sol_b = unrolled(tls, 14)
    diff = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(ga, gb))
    print(f"loss {float(loss_b):.16e}; gradient change 12 -> 14 steps: {diff:.3e}")
    np.savez(os.path.join(HERE, "adjoint_small.npz"), loss=float(loss_b), grad_uv_free=gb[0].numpy(),
             grad_uv_fixed=gb[1].numpy(), cams=sol_b["cams"].numpy(), points=sol_b["points"].numpy(),
             unroll_change=diff)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCHLS_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the torchls checkout> "
                 "(or set TORCHLS_REFERENCE)")
    main(ref)
