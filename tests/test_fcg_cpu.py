"""CPU check of the flexible-CG restatement (tests/fcg_ref.py) on the oracle:
it reaches 1e-10 on the heterogeneous, anisotropic generator where the plain
cycle stalls, its recurrence residual matches the true residual, and with a
symmetric cycle (V(1,1)) the preconditioner is symmetric to rounding."""
import numpy as np

from cedar_b200 import gallery as G
from cedar_b200 import problems as P
from tests.fcg_ref import fcg


def test_fcg_reference_converges_where_plain_cycle_stalls(oracle):
    n = 63
    so, b = P.hetero_diffusion(n)
    _, h_plain = oracle.Solver(so, relax="line-xy", maxiter=40, tol=1e-10).solve(b)
    assert h_plain[-1] > 1e-3
    x, h, true_rel = fcg(oracle, so, b, tol=1e-6)
    assert h[-1] < 1e-6 and len(h) < 60
    assert true_rel < 1e-6
    r = oracle.residual(np.ascontiguousarray(so), x, b)
    assert np.linalg.norm(r) / np.linalg.norm(b[1:-1, 1:-1]) < 1e-6


def test_hetero_generator_fp64_floor_is_above_1e10():
    """On the heterogeneous, anisotropic generator (1e4 inclusions on a sigma = 2
    lognormal field, anisotropy 1e-3) a relative residual of 1e-10 lies below
    what FP64 arithmetic can attain: a sparse direct solve stops near 1e-8, and
    eps * |A||x| / |b| (the rounding of the residual itself) is of that size.
    Without the inclusions and the anisotropy the floor drops near 1e-11."""
    import scipy.sparse.linalg as spla
    for kw, lo, hi in (({}, 1e-9, 1e-6), ({"contrast": 1.0, "aniso": 1.0}, 1e-13, 2e-10)):
        so, b = P.hetero_diffusion(127, **kw)
        A = G.stencil_to_csr(so).tocsc()
        bv = b[1:-1, 1:-1].ravel()
        x = spla.spsolve(A, bv)
        direct = np.linalg.norm(bv - A @ x) / np.linalg.norm(bv)
        floor = np.finfo(float).eps * np.linalg.norm(abs(A) @ abs(x)) / np.linalg.norm(bv)
        assert lo < direct < hi and lo < floor < 10 * hi, (kw, direct, floor)


def test_symmetric_cycle_is_a_symmetric_preconditioner(oracle):
    n = 31
    so, _ = P.hetero_diffusion(n)
    pre = oracle.Solver(so, relax="line-xy", maxiter=1, tol=1e-300, nrelax_pre=1, nrelax_post=1)
    rng = np.random.default_rng(5)

    def M(v):
        rr = np.zeros((n + 2, n + 2))
        rr[1:-1, 1:-1] = v.reshape(n, n)
        z, _ = pre.solve(rr)
        return z[1:-1, 1:-1].ravel()

    u, v = rng.standard_normal(n * n), rng.standard_normal(n * n)
    assert abs(u @ M(v) - v @ M(u)) <= 1e-10 * abs(u @ M(v))
    A = G.stencil_to_csr(so)
    assert u @ M(A @ u) > 0
