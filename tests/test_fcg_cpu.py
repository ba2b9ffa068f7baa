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


def test_oracle_fcg_matches_python_restatement(oracle):
    """The oracle's C flexible CG (the CPU baseline's solver) follows the numpy
    restatement over the same cycle: same iteration count, histories equal to
    rounding (the two sum their dot products in different orders), and with
    residual replacement (formed every 4th iteration) the same tolerance."""
    n = 63
    so, b = P.hetero_diffusion(n)
    x_ref, h_ref, _ = fcg(oracle, so, b, tol=1e-6, num_levels=3)
    s = oracle.Solver(so, relax="line-xy", nrelax_pre=1, nrelax_post=1, num_levels=3, maxiter=200, tol=1e-6)
    x, h = s.solve_fcg(b)
    assert len(h) == len(h_ref)
    np.testing.assert_allclose(h[:10], h_ref[:10], rtol=1e-7)
    assert np.abs(x - x_ref).max() <= 1e-6 * np.abs(x_ref).max()
    x4, h4 = oracle.Solver(so, relax="line-xy", nrelax_pre=1, nrelax_post=1, num_levels=3, maxiter=200,
                           tol=1e-6).solve_fcg(b, replace=4)
    r = oracle.residual(np.ascontiguousarray(so), x4, b)
    r0 = oracle.residual(np.ascontiguousarray(so), np.zeros_like(b), b)
    assert h4[-1] < 1e-6 and np.linalg.norm(r) / np.linalg.norm(r0) < 1e-6
    assert abs(len(h4) - len(h)) <= 3
    np.testing.assert_allclose(h4[:3], h[:3], rtol=1e-7)


def test_oracle_fcg_thread_count_independent(oracle):
    """Row partials summed in row order: one host thread and four give the same bits."""
    n = 767
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
    out = []
    for t in (1, 4):
        oracle.set_threads(t)
        try:
            s = oracle.Solver(so, relax="line-xy", nrelax_pre=1, nrelax_post=1, num_levels=4, maxiter=3, tol=0.0)
            out.append(s.solve_fcg(b))
        finally:
            oracle.set_threads(0)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
