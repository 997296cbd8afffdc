"""CPU oracle for the block-sparse LM/GN inner loop -- TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of the torchls algorithm for the LM/GN path
(linearize -> gradient -> diagonal blocks -> block-Jacobi -> PCG / Schur-PCG /
dense Schur -> retract -> trial cost). Each function cites the torchls
file:line it restates.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or as the timed CPU
baseline; the CUDA product path never calls into it.

Parity pins: ``tests/golden/`` holds fixtures produced by running torchls
itself (float64, CPU) on the seeded synthetic problems; ``tests/test_oracle.py``
checks this restatement against them.

Linearization of residual functions that have no analytic numpy form here is
done the way torchls does it -- ``torch.func.vmap(jacrev)`` of the residual
through the retraction's first-order chart, on CPU in float64 -- because the
residual function itself is user code, not part of the algorithm under test.
"""

from .model import OracleProblem, huber_loss  # noqa: F401
from .lm import solve  # noqa: F401
