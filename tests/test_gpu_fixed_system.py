"""FixedLinearSystem / LinearFactor / least_absolute_deviations on the GPU
against torchls's own (linear_system.py:15-141), from ``fixed_system.npz``:
products and solves within 1e-11 relative, the LAD ADMM path (one run that
converges, one cut at 60 iterations) within 1e-8 with the same iteration
count, and the reference's validation errors."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from gpu_helpers import close, load, needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _system(tls):
    fx = load("fixed_system")
    t = lambda k: torch.from_numpy(fx[k]).to(DEV)  # noqa: E731
    return fx, t, tls.FixedLinearSystem(t("A").to_sparse())


def test_products_factor_and_solve():
    import torchls_b200 as tls

    fx, t, fs = _system(tls)
    close(fs.matvec(t("x")), fx["matvec"], 1e-12, what="matvec")
    close(fs.matvec(t("x")[:, 0]), fx["matvec1"], 1e-12, what="matvec (one column)")
    close(fs.rmatvec(t("y")), fx["rmatvec"], 1e-12, what="rmatvec")
    fac = fs.factor(t("w"), ridge=0.1)
    close(fac.cholesky, fx["cholesky"], 1e-11, what="weighted normal factor")
    close(fac.least_squares(t("target")), fx["weighted_ls"], 1e-11, what="weighted least squares")
    close(fs.factor().solve(t("x")), fx["solve"], 1e-11, what="solve")


def test_least_absolute_deviations():
    import torchls_b200 as tls

    fx, t, fs = _system(tls)
    res = tls.least_absolute_deviations(fs, t("target"), rho=0.3, max_iterations=200)
    assert res.converged == bool(fx["lad_converged"]) and res.iterations == int(fx["lad_iterations"])
    close(res.solution, fx["lad_solution"], 1e-8, what="LAD solution")
    res1 = tls.least_absolute_deviations(fs, t("target")[:, 0], rho=1.0, max_iterations=60)
    assert res1.iterations == int(fx["lad1_iterations"]) and not res1.converged
    close(res1.solution, fx["lad1_solution"], 1e-8, what="LAD solution (one column, capped)")


def test_validation_errors():
    import torchls_b200 as tls

    fx, t, fs = _system(tls)
    with pytest.raises(ValueError, match="max_dense_columns"):
        tls.FixedLinearSystem(t("A"), max_dense_columns=10)
    with pytest.raises(ValueError, match="ridge"):
        fs.factor(ridge=-1.0)
    with pytest.raises(ValueError, match="weights"):
        fs.factor(-t("w"))
    with pytest.raises(ValueError, match="incompatible"):
        fs.matvec(t("y"))
    with pytest.raises(ValueError, match="unweighted"):
        tls.least_absolute_deviations(fs, t("target"), factor=fs.factor(t("w")))
    with pytest.raises(ValueError):
        tls.FixedLinearSystem(torch.tensor([[float("nan")]], dtype=torch.float64, device=DEV))
    assert np.isfinite(fx["lad_solution"]).all()
