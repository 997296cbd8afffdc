"""The typed API's analysis on the host: ``LeastSquaresProblem.analyze`` over
``Cost.factory`` costs and ``Var`` handles with sparse, unsorted IDs gives the
reference's layout (group order as declared, IDs sorted, offsets cumulative),
pinned by ``typed_ba.npz`` written by torchls itself."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from golden import problems as P
from test_oracle import load


def test_typed_layout_matches_reference():
    import torchls_b200 as tls

    fx = load("typed_ba")
    problem, init = P.typed_ba(tls)
    np.testing.assert_array_equal([e.offset for e in problem.layout], fx["offsets"])
    np.testing.assert_array_equal([e.dim for e in problem.layout], fx["dims"])
    for i, e in enumerate(problem.layout):
        np.testing.assert_array_equal(e.ids.numpy(), fx[f"ids{i}"])
        assert torch.equal(init._ids[e.key], e.ids)


def test_typed_api_validation():
    import torchls_b200 as tls

    class Q(tls.Var, default_factory=lambda: torch.zeros(2)):
        pass

    with pytest.raises(ValueError, match="unique"):
        tls.LeastSquaresProblem([tls.Cost(lambda q: q, (Q(torch.tensor([1, 1])),))],
                                [Q(torch.tensor([1, 1]))]).analyze()
    with pytest.raises(ValueError, match="in_dims"):
        tls.Cost(lambda q: q, (Q(1),), in_dims=(1,))
    with pytest.raises(ValueError, match="batch_size"):
        tls.Cost(lambda q: q, (Q(1),), batch_size=0)
    with pytest.raises(ValueError, match="sorted and unique"):
        tls.VarValues({Q: torch.zeros(2, 2)}, {Q: torch.tensor([2, 1])})
    with pytest.raises(ValueError, match="expected shape"):
        tls.VarValues.make([Q(torch.tensor([1, 2])).with_value(torch.zeros(3, 2))])
    vals = tls.VarValues.make([Q(torch.tensor([5, 2])).with_value(torch.tensor([[5.0, 5.0], [2.0, 2.0]]))])
    assert vals[Q(5)].tolist() == [5.0, 5.0] and vals[Q].shape == (2, 2)
    with pytest.raises(KeyError):
        vals[Q(3)]
