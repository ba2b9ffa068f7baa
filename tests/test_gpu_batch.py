"""Batches of independent 2D problems solved together (cdr_gpu_batch2d_*).

Every problem must end where its own solve would: with the sequential line
substitutions the FP64 batch reproduces the oracle's iterates bit for bit and
stops each problem at the oracle's cycle; the FP32-refined batch gives each
problem the iterate of a single-problem FP32-refined solve.
"""
import numpy as np
import pytest

from cedar_b200 import gallery as G
from cedar_b200 import problems as P
from cedar_b200.config import Config
from tests.gpu_util import host

pytestmark = pytest.mark.gpu


def _batch(nx, ny, nb, ns, seed):
    ops, rhs = [], []
    for p in range(nb):
        if ns == 5:
            kx, ky = P.hetero_coefficients(max(nx, ny), sigma=1.0 + 0.2 * p, n_incl=4, contrast=100.0, aniso=0.5,
                                           seed_field=seed + p, seed_incl=seed + 50 + p)
            so = G.fe_hetero(kx[:ny + 1, :nx + 1], ky[:ny + 1, :nx + 1])
        else:
            so = G.diag_diffusion(nx, ny, 1.0 + p, 0.5)
        rng = np.random.default_rng(seed + 100 + p)
        b = np.zeros((ny + 2, nx + 2))
        b[1:-1, 1:-1] = rng.uniform(0, 1, (ny, nx)) / (nx + 1) ** 2
        ops.append(np.ascontiguousarray(so))
        rhs.append(b)
    return ops, rhs


def _device(arrs, pitch):
    import torch
    a = np.stack(arrs)
    out = torch.zeros(a.shape[:-1] + (pitch,), dtype=torch.float64, device="cuda")
    out[..., :a.shape[-1]] = torch.from_numpy(a).cuda()
    return out


def _solve_batch(ops, rhs, conf):
    from cedar_b200.solver import BatchSolver2D
    ns, jj, ii = ops[0].shape
    nx, ny = ii - 2, jj - 2
    pitch = ((ii + 7) // 8) * 8
    so, b = _device(ops, pitch), _device(rhs, pitch)
    x = b.clone().zero_()
    s = BatchSolver2D(so.data_ptr(), ns, nx, ny, pitch, len(ops), conf)
    s.solve_device(b.data_ptr(), x.data_ptr())
    return host(x)[..., :ii], s


@pytest.mark.parametrize("relax,ns", [("line-xy", 5), ("point", 3), ("point", 5)])
def test_batch_fp64_matches_oracle_per_problem(oracle, relax, ns):
    nx, ny, nb = 47, 33, 5
    ops, rhs = _batch(nx, ny, nb, ns, seed=30)
    conf = Config({"solver": {"relaxation": relax, "max-iter": 30, "tol": 1e-9},
                   "gpu": {"line-solve": "sequential"}})
    x, s = _solve_batch(ops, rhs, conf)
    for p in range(nb):
        xr, hr = oracle.Solver(ops[p], relax=relax, maxiter=30, tol=1e-9).solve(rhs[p])
        assert s.iters[p] == len(hr), "problem %d: %d cycles vs %d" % (p, s.iters[p], len(hr))
        assert abs(s.rel[p] - hr[-1]) <= 1e-12 * max(1.0, abs(hr[-1]))
        assert np.array_equal(x[p], xr), "problem %d differs" % p
    assert np.all(s.done_ms > 0)


def test_batch_fp32_ir_matches_single_solves():
    """Each problem of an FP32-refined batch converges like a single-problem
    FP32-refined solve: same tolerance, cycle counts within one, iterates equal
    to 1e-7 relative (the FP64 refinement pins them; the FP32 cycles differ in
    rounding, since single problems and batches have different default line
    shapes on short lines)."""
    from cedar_b200.solver import Solver2D
    nx, ny, nb = 63, 63, 4
    ops, rhs = _batch(nx, ny, nb, 5, seed=40)
    conf = Config({"solver": {"relaxation": "line-xy", "cycle": {"nrelax-pre": 1, "nrelax-post": 1},
                              "max-iter": 40, "tol": 1e-8}, "gpu": {"precision": "fp32-ir", "autotune": False}})
    x, s = _solve_batch(ops, rhs, conf)
    for p in range(nb):
        single = Solver2D(ops[p], conf)
        xs = single.solve(rhs[p])
        assert s.rel[p] < 1e-8 and single.history[-1] < 1e-8
        assert abs(single.iters - s.iters[p]) <= 1
        assert np.abs(x[p] - xs).max() <= 1e-7 * np.abs(xs).max()


def test_batch_rejects_bad_arguments():
    import ctypes
    from cedar_b200 import _lib
    lib = _lib.load()
    st = _lib.Settings()
    lib.cdr_gpu_settings_default(ctypes.byref(st))
    h = ctypes.c_void_p()
    assert lib.cdr_gpu_batch2d_create(ctypes.byref(st), None, 5, 9, 9, 16, 2, None, ctypes.byref(h)) == 1
    st.relaxation = 7  # a 3D smoother
    assert lib.cdr_gpu_batch2d_create(ctypes.byref(st), ctypes.c_void_p(16), 5, 9, 9, 16, 2, None,
                                      ctypes.byref(h)) == 1
