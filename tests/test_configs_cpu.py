"""Config surface (solvers.py:19-164 of the reference): the reference's
backend names construct unchanged, unknown names and bad values raise."""

from __future__ import annotations

import pytest


def test_reference_backend_names_are_accepted():
    import torchls_b200 as tls

    for backend in ("cuda", "torch", "warp"):
        cfg = tls.ConjugateGradientConfig(backend=backend, normal_matvec=backend)
        assert cfg.backend == backend
    with pytest.raises(ValueError, match="backend"):
        tls.ConjugateGradientConfig(backend="cpu")
    with pytest.raises(ValueError, match="normal_matvec"):
        tls.ConjugateGradientConfig(normal_matvec="numpy")


def test_config_validation():
    import torchls_b200 as tls

    with pytest.raises(ValueError):
        tls.ConjugateGradientConfig(rtol=-1)
    with pytest.raises(ValueError):
        tls.ConjugateGradientConfig(preconditioner_groups=(("a",),))
    with pytest.raises(ValueError):
        tls.TrustRegionConfig(lambda_initial=0)
    with pytest.raises(ValueError):
        tls.TerminationConfig(target_cost=float("nan"))
    with pytest.raises(ValueError):
        tls.ConjugateGradientConfig(precision="half")
