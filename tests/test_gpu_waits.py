"""The bounded waits of the two streamed kernels and how a give-up is reported.

The streamed x-line sweep and the explicit-inverse coarsest product wait on
their own bulk copies (mbarrier phases).  A CTA that gives up counts itself,
waits for the copies it still has in flight and leaves; the status call and
the solver then return CDR_ERR_NUMERIC and reset the count.  Two checks:
the host path alone (counts injected from the host, no device wait), and the
device path with the wait limit set to zero, which makes every CTA give up
at its first wait, on copies that have only just been issued.  The copies
themselves complete, so every drain ends; the limit is restored afterwards and
the same calls run clean again on the same context.
"""
import ctypes

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import gallery as G
from cedar_b200 import problems as P
from cedar_b200.config import Config
from tests.gpu_util import host, padded, ptr, stream

pytestmark = pytest.mark.gpu
NUMERIC = 6


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    L = _lib.load()
    yield L
    L.cdr_gpu_set_wait_limit_ns(-1)


def _xline_problem(n=511):
    import torch
    rng = np.random.default_rng(3)
    so = np.ascontiguousarray(G.fe_hetero(np.exp(rng.standard_normal((n + 1, n + 1))),
                                          np.exp(rng.standard_normal((n + 1, n + 1)))))
    x = np.zeros((n + 2, n + 2))
    x[1:-1, 1:-1] = rng.standard_normal((n, n))
    b = np.zeros_like(x)
    b[1:-1, 1:-1] = rng.standard_normal((n, n))
    from oracle import oracle as O
    O.build()
    sx, _ = O.setup_lines_x(so)
    gx = sx.copy()
    gx[0][1:-1, 1:-1] = 1.0 / sx[0][1:-1, 1:-1]
    pitch = ((n + 2 + 31) // 32) * 32
    f = torch.float32
    return n, pitch, padded(so, pitch, f), padded(x, pitch, f), padded(b, pitch, f), padded(gx, pitch, f), x


def test_injected_counts_are_reported_and_reset(lib):
    """Host path: a count in either give-up counter turns into CDR_ERR_NUMERIC
    at the next status check, which resets it."""
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0
    _lib.check(lib.cdr_gpu_inject_timeouts(3, 0))
    assert lib.cdr_gpu_lines_stream_status(stream()) == NUMERIC
    assert b"gave up" in lib.cdr_gpu_last_error()
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0
    # the solver reads both counters after every solve
    from cedar_b200.solver import Solver2D
    so, b = P.hetero_diffusion(255, sigma=1.0, n_incl=0, aniso=1.0)
    s = Solver2D(so, Config({"solver": {"relaxation": "line-xy", "num-levels": 3, "max-iter": 3, "tol": 1e-12},
                             "gpu": {"coarse-solve": "inverse"}}))
    s.solve(b)
    for lines, inverse in ((1, 0), (0, 2), (4, 5)):
        _lib.check(lib.cdr_gpu_inject_timeouts(lines, inverse))
        with pytest.raises(_lib.CdrError) as e:
            s.solve(b)
        assert e.value.code == NUMERIC
        s.solve(b)  # reset: the next solve is clean


def test_streamed_x_line_give_up(lib):
    """Device path: with the wait limit at zero, every CTA of the streamed
    x-line kernel gives up on the rows it has just requested; the
    sweep reports CDR_ERR_NUMERIC.  With the default limit restored the same
    sweep is clean and equals the register-chunk kernel bit for bit."""
    n, pitch, dso, dx0, dbb, dsx, _ = _xline_problem()
    args = lambda dx, flags: (ptr(dso), 5, ptr(dx), ptr(dbb), ptr(dsx), n, n, pitch, pitch, _lib.DIR_X, 0, flags,
                              stream())
    _lib.check(lib.cdr_gpu_set_wait_limit_ns(0))
    try:
        dx = dx0.clone()
        _lib.check(lib.cdr_gpu_relax_lines_2d_f32(*args(dx, _lib.LINES_STREAM)))
        assert lib.cdr_gpu_lines_stream_status(stream()) == NUMERIC
    finally:
        _lib.check(lib.cdr_gpu_set_wait_limit_ns(-1))
    dx = dx0.clone()
    _lib.check(lib.cdr_gpu_relax_lines_2d_f32(*args(dx, _lib.LINES_STREAM)))
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0
    dref = dx0.clone()
    _lib.check(lib.cdr_gpu_relax_lines_2d_f32(*args(dref, _lib.LINES_NOTUNE)))
    np.testing.assert_array_equal(host(dx), host(dref))


def test_inverse_product_give_up(lib):
    """Device path of the explicit-inverse coarsest product (64^2 coarsest
    level, rows streamed into shared memory): a solve with the wait limit at
    zero fails with CDR_ERR_NUMERIC; with the default limit
    the same handle solves to the tolerance."""
    from cedar_b200.solver import Solver2D
    so, b = P.hetero_diffusion(255, sigma=1.0, n_incl=0, aniso=1.0)
    s = Solver2D(so, Config({"solver": {"relaxation": "line-xy", "num-levels": 3, "max-iter": 30, "tol": 1e-9},
                             "gpu": {"coarse-solve": "inverse", "graph": False}}))
    _lib.check(lib.cdr_gpu_set_wait_limit_ns(0))
    try:
        with pytest.raises(_lib.CdrError) as e:
            s.solve(b)
        assert e.value.code == NUMERIC
    finally:
        _lib.check(lib.cdr_gpu_set_wait_limit_ns(-1))
    s.solve(b)
    assert s.history[-1] < 1e-9
