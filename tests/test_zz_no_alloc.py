"""``tls_squared_matvec_norm_static``: |J x|^2 without a caller scratch buffer.

Some callers cannot allocate device memory where they need this norm (code
inside another framework's memory pool, a binding with no device allocator,
a loop where an allocation may block). This entry point keeps its block
partials in an array inside the library instead. The test calls it through
the C ABI twice in a row and compares each result with the buffer-taking
``tls_squared_matvec_norm`` (1e-12 relative, the tolerance of the other
product tests), then checks that an oversized factor group is rejected
before any work, as are a column scale whose dtype is not float64 and null
pointers.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from gpu_helpers import close, load, needs_gpu, stored_ba
from golden import problems as P

pytestmark = [pytest.mark.gpu, needs_gpu]

DEV = "cuda"


def _static_norm(L, args, x):
    out = torch.full((), float("nan"), dtype=torch.float64, device=x.device)
    L.call("tls_squared_matvec_norm_static", ctypes.byref(args), x.data_ptr(), out.data_ptr(),
           L.stream_handle(x.device))
    return out


def test_static_squared_norm_matches_buffered_entry_point():
    import torchls_b200 as tls
    from torchls_b200 import _lib as L

    fx = load("ba_small")
    J = P.ba_small(tls, device=DEV, data=stored_ba(fx)).linearize().jacobian
    v = torch.from_numpy(fx["v"]).to(DEV)
    gen = torch.Generator().manual_seed(3)
    w = torch.randn(v.shape, generator=gen, dtype=torch.float64).to(DEV)
    for jac, vec in ((J, v), (J, w), (J.scale_columns(1.0 + w.abs()), v)):
        args = jac.normal_args(torch.float64)
        want = jac.squared_matvec_norm(vec)  # buffer-taking entry point
        first = _static_norm(L, args, vec)
        second = _static_norm(L, args, vec)
        torch.cuda.synchronize()
        close(first, want, 1e-12, what="first call")
        close(second, want, 1e-12, what="second call")
        assert torch.equal(first, second), "two calls in a row differ"
    close(_static_norm(L, J.normal_args(torch.float64), v), fx["squared_matvec_norm"], 1e-12, what="fixture")


def test_static_squared_norm_rejects_oversized_groups():
    from torchls_b200 import _lib as L

    args = L.NormalArgs()
    args.nfactor_groups = 1
    args.fg[0].count = 65536 * 128 + 1  # checked on the host before any device work
    args.fg[0].rdim = 2
    out = torch.zeros((), dtype=torch.float64, device=DEV)
    x = torch.zeros(8, dtype=torch.float64, device=DEV)
    before = L.launch_count()
    with pytest.raises(ValueError, match="8,388,608"):
        L.call("tls_squared_matvec_norm_static", ctypes.byref(args), x.data_ptr(), out.data_ptr(),
               L.stream_handle(x.device))
    assert L.launch_count() == before
    assert np.isfinite(float(out))


def test_static_squared_norm_rejects_bad_arguments():
    from torchls_b200 import _lib as L

    args = L.NormalArgs()
    args.nfactor_groups = 0
    args.vec_dtype = L.dtype_code(torch.float32)
    scale = torch.ones(8, dtype=torch.float32, device=DEV)
    args.scale = scale.data_ptr()  # read as float64 by the kernel: must be refused
    out = torch.zeros((), dtype=torch.float64, device=DEV)
    x = torch.zeros(8, dtype=torch.float64, device=DEV)
    before = L.launch_count()
    with pytest.raises(ValueError, match="float64"):
        L.call("tls_squared_matvec_norm_static", ctypes.byref(args), x.data_ptr(), out.data_ptr(),
               L.stream_handle(x.device))
    with pytest.raises(ValueError, match="null"):
        L.call("tls_squared_matvec_norm_static", ctypes.byref(args), None, out.data_ptr(),
               L.stream_handle(x.device))
    with pytest.raises(ValueError, match="null"):
        L.call("tls_squared_matvec_norm_static", None, x.data_ptr(), out.data_ptr(), L.stream_handle(x.device))
    assert L.launch_count() == before
