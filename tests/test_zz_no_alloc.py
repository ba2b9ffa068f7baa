"""The allocation-free residual entry point.

Some callers cannot allocate device memory when they call this library (a
plugin inside an application that owns every device allocation and forbids
cudaMalloc/cudaFree during a run).  cdr_gpu_residual_2d_f64_noalloc computes
r = b - A x and ||r||_2 with its partial sums in a fixed device array instead of
caller scratch.  This file checks, through the C ABI, that two calls in a row
give the same r (bit for bit) and the same norm (1e-13 relative; the partial
sums are grouped per tile instead of per block) as the regular entry point, and
that grids beyond the array's capacity are refused, and that calls after
the first leave the device's free memory unchanged.  It is collected last.
"""
import ctypes

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import problems as P
from tests.gpu_util import host, padded, ptr, stream

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    return _lib.load()


@pytest.mark.parametrize("n,ns,pad", [(2047, 5, True), (1000, 3, True), (9, 5, False), (513, 5, False)])
def test_noalloc_matches_allocating_residual_twice(lib, n, ns, pad):
    import torch
    if ns == 5:
        so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=8, contrast=100.0, aniso=0.1)
    else:
        so, b = P.poisson_noise(n)
    pitch = ((n + 2 + 31) // 32) * 32 if pad else n + 2
    dso, db = padded(so, pitch), padded(b, pitch)
    scratch = torch.zeros(lib.cdr_gpu_norm_scratch_bytes() // 8, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(n)
    for call in range(2):
        x = np.zeros((n + 2, n + 2))
        x[1:-1, 1:-1] = rng.standard_normal((n, n)) * (call + 1)
        dx = padded(x, pitch)
        r_ref = torch.zeros_like(dx)
        r_new = torch.full_like(dx, float("nan"))
        r_new[0, :] = 0.0; r_new[-1, :] = 0.0; r_new[:, 0] = 0.0; r_new[:, n + 1:] = 0.0
        nrm_ref = torch.zeros(1, dtype=torch.float64, device="cuda")
        nrm_new = torch.zeros(1, dtype=torch.float64, device="cuda")
        _lib.check(lib.cdr_gpu_residual_2d_f64(ptr(dso), ns, ptr(dx), ptr(db), ptr(r_ref), n, n, pitch, ptr(nrm_ref),
                                               ptr(scratch), stream()))
        _lib.check(lib.cdr_gpu_residual_2d_f64_noalloc(ptr(dso), ns, ptr(dx), ptr(db), ptr(r_new), n, n, pitch,
                                                       ptr(nrm_new), stream()))
        np.testing.assert_array_equal(host(r_new)[:, :n + 2], host(r_ref)[:, :n + 2])
        a, e = host(nrm_new)[0], host(nrm_ref)[0]
        assert np.isfinite(a) and abs(a - e) <= 1e-13 * e, (call, a, e)


def test_noalloc_calls_allocate_no_device_memory(lib):
    """After a first call (which looks up the array's address), further calls
    leave the device's free memory unchanged: nothing is allocated."""
    import torch
    n = 1023
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=8, contrast=100.0, aniso=0.1)
    pitch = ((n + 2 + 31) // 32) * 32
    dso, db = padded(so, pitch), padded(b, pitch)
    dx = padded(np.zeros_like(b), pitch)
    dr = torch.zeros_like(dx)
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.check(lib.cdr_gpu_residual_2d_f64_noalloc(ptr(dso), 5, ptr(dx), ptr(db), ptr(dr), n, n, pitch, ptr(nrm),
                                                   stream()))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        _lib.check(lib.cdr_gpu_residual_2d_f64_noalloc(ptr(dso), 5, ptr(dx), ptr(db), ptr(dr), n, n, pitch,
                                                       ptr(nrm), stream()))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_grids_beyond_its_scratch(lib):
    import torch
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.cdr_gpu_residual_2d_f64_noalloc(ptr(t), 5, ptr(t), ptr(t), ptr(t), 4097, 4097, 4128, ptr(t), stream())
    assert rc == 2  # CDR_ERR_DIM, nothing launched
    assert b"65536" in lib.cdr_gpu_last_error()
    rc = lib.cdr_gpu_residual_2d_f64_noalloc(ptr(t), 5, ptr(t), ptr(t), ptr(t), 4096, 4096, 4098, None, stream())
    assert rc == 1  # CDR_ERR_ARG: the norm output is required
