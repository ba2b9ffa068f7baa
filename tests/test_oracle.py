"""CPU tests of the parity oracle (oracle/cdr2_oracle.c) against the reference's
published golden output, LAPACK, and algebraic identities.  No GPU."""
import json
import os

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from cedar_b200 import gallery as G
from cedar_b200 import problems as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_readme_history_pinned(oracle):
    """Residual history of README.md:49-63 to the 6 printed digits, all 10 iterations."""
    g = json.load(open(os.path.join(GOLD, "readme_poisson400.json")))
    so = G.poisson(400, 400)
    b = G.poisson_rhs_sin2pi(400, 400)
    s = oracle.Solver(so, relax="point", nrelax_pre=1, nrelax_post=1, maxiter=10, tol=1e-10,
                      num_levels=g["num_levels"])
    x, h = s.solve(b)
    assert len(h) == 10
    for got, ref in zip(h, g["history"]):
        assert float("%.6g" % got) == ref
    err = oracle.inf_norm(np.ascontiguousarray(G.poisson_exact_sin2pi(400, 400) - x))
    assert float("%.6g" % abs(err)) == g["solution_norm_abs"]


def test_serial_level_rule(oracle):
    """compute_num_levels of include/cedar/2d/solver.h:63-79 (min_coarse 3)."""
    assert oracle.num_levels(400, 400, 3) == 8
    assert oracle.num_levels(511, 511, 3) == 8
    assert oracle.num_levels(2047, 2047, 3) == 10
    assert oracle.num_levels(1023, 1023, 3) == 9
    assert oracle.num_levels(63, 63, 3) == 5
    s = oracle.Solver(G.poisson(400, 400))
    assert [s.level_dims(l)[0] for l in range(s.nlevels)] == [400, 200, 100, 50, 25, 13, 7, 4]


def test_oracle_fixture_histories(oracle):
    """Regression pin of the oracle on small cases (fixtures written by make_fixtures.py)."""
    fx = json.load(open(os.path.join(GOLD, "oracle_histories.json")))
    from tests.golden.make_fixtures import build_case
    for case in fx["cases"]:
        so, b, kw = build_case(case)
        s = oracle.Solver(so, **kw)
        x, h = s.solve(b)
        np.testing.assert_allclose(h, case["history"], rtol=1e-13, atol=0)


def test_dpttrf_dpttrs_match_lapack(oracle):
    rng = np.random.default_rng(0)
    for n in (2, 5, 37, 200):
        d = 4 + rng.random(n)
        e = -rng.random(max(n - 1, 0))
        d1, e1, info = oracle.dpttrf(d, e)
        d2, e2, info2 = lapack.dpttrf(d, e)[:3]
        assert info == info2 == 0
        np.testing.assert_array_equal(d1, d2)
        np.testing.assert_array_equal(e1, e2)
        bb = rng.random(n)
        np.testing.assert_array_equal(oracle.dpttrs(d1, e1, bb), lapack.dpttrs(d2, e2, bb)[0])


def test_dpttrf_reports_nonpositive_pivot(oracle):
    d, e, info = oracle.dpttrf([1.0, 1.0, 1.0], [-2.0, 0.0])
    assert info == 2


def test_dpbtrf_dpbtrs_match_lapack(oracle):
    rng = np.random.default_rng(1)
    for N, kd in ((16, 5), (64, 21), (9, 4)):
        A = np.zeros((N, N))
        for i in range(N):
            A[i, i] = 2 * kd + 1 + rng.random()
            for k in range(1, kd + 1):
                if i + k < N:
                    A[i, i + k] = A[i + k, i] = -rng.random()
        ab = np.zeros((kd + 1, N))
        for j in range(N):
            for i in range(max(0, j - kd), j + 1):
                ab[kd + i - j, j] = A[i, j]
        f1, info = oracle.dpbtrf_u(ab, kd)
        f2, info2 = lapack.dpbtrf(ab, lower=0)
        assert info == info2 == 0
        np.testing.assert_allclose(f1, f2, rtol=1e-14, atol=1e-14)
        b = rng.random(N)
        np.testing.assert_allclose(oracle.dpbtrs_u(f1, kd, b), np.linalg.solve(A, b), rtol=1e-12)


def test_coarse_solve_is_exact_inverse(oracle):
    so = G.fe_hetero(*P.hetero_coefficients(5, n_incl=2))
    abd, info = oracle.setup_cg(so)
    assert info == 0
    rng = np.random.default_rng(2)
    b = np.zeros((7, 7))
    b[1:-1, 1:-1] = rng.random((5, 5))
    x = oracle.solve_cg(abd, b)
    A = G.stencil_to_csr(so).toarray()
    np.testing.assert_allclose(x[1:-1, 1:-1].ravel(), np.linalg.solve(A, b[1:-1, 1:-1].ravel()), rtol=1e-12)


@pytest.mark.parametrize("nx,ny,ns", [(9, 9, 3), (10, 8, 3), (9, 12, 5), (12, 11, 5), (8, 8, 5), (15, 14, 5)])
def test_galerkin_equals_ptap(oracle, nx, ny, ns):
    """ITLI coarse operator == P^T A P assembled from the interpolation as interp_add applies it."""
    rng = np.random.default_rng(nx * 100 + ny)
    if ns == 3:
        so = G.diag_diffusion(nx, ny, 1.0, 0.3)
        so[1:] *= 1 + 0.3 * rng.random(so[1:].shape)
        so[:, 0, :] = 0; so[:, :, 0] = 0
        so[1, :, 1] = 0; so[2, 1, :] = 0
    else:
        kx = np.exp(rng.normal(size=(ny + 1, nx + 1)))
        so = G.fe_hetero(kx, kx * np.exp(rng.normal(size=(ny + 1, nx + 1))))
    nxc, nyc = (nx - 1) // 2 + 1, (ny - 1) // 2 + 1
    ci = oracle.setup_interp(so, nxc, nyc)
    soc = oracle.galerkin(so, ci)
    # explicit P from interp_add applied to unit coarse vectors
    A = G.stencil_to_csr(so).toarray()
    Pm = np.zeros((nx * ny, nxc * nyc))
    for jc in range(nyc):
        for ic in range(nxc):
            xc = np.zeros((nyc + 2, nxc + 2))
            xc[jc + 1, ic + 1] = 1.0
            xf = np.zeros((ny + 2, nx + 2))
            oracle.interp_add(ci, xc, np.zeros_like(xf), np.ascontiguousarray(so), xf)
            Pm[:, jc * nxc + ic] = xf[1:-1, 1:-1].ravel()
    Ac = Pm.T @ A @ Pm
    Acs = G.stencil_to_csr(soc).toarray()
    assert np.abs(Ac - Acs).max() <= 1e-13 * np.abs(Ac).max()


def test_restrict_is_transpose_of_interp(oracle):
    nx = ny = 13
    so = G.fe_hetero(*P.hetero_coefficients(nx, n_incl=3))
    ci = oracle.setup_interp(so, 7, 7)
    rng = np.random.default_rng(5)
    r = np.zeros((ny + 2, nx + 2)); r[1:-1, 1:-1] = rng.random((ny, nx))
    xc = np.zeros((9, 9)); xc[1:-1, 1:-1] = rng.random((7, 7))
    bc = oracle.restrict(ci, r)
    xf = np.zeros_like(r)
    oracle.interp_add(ci, xc, np.zeros_like(r), np.ascontiguousarray(so), xf)
    assert abs((bc * xc).sum() - (r * xf).sum()) < 1e-12 * abs((r * xf).sum())


def test_gallery_fe_matches_hetero_constant():
    n = 11
    so = G.fe_hetero(np.ones((n + 1, n + 1)), np.ones((n + 1, n + 1))) * 3
    np.testing.assert_allclose(so, G.fe(n, n), atol=1e-15)


def test_hetero_operator_symmetric_positive():
    n = 15
    so = G.fe_hetero(*P.hetero_coefficients(n))
    A = G.stencil_to_csr(so).toarray()
    assert np.abs(A - A.T).max() == 0
    assert np.linalg.eigvalsh(A).min() > 0


def test_line_smoothers_converge_like_reference_tests(oracle):
    """test/2d/test_poisson.cc:96-159 thresholds: line-x on 800x200-shaped and line-y on
    200x800-shaped anisotropic problems reach ||r|| < 1e-8 (scaled down here)."""
    for relax, (nx, ny), (dx, dy) in (("line-x", (160, 40), (1.0, 1e-3)), ("line-y", (40, 160), (1e-3, 1.0))):
        so = G.diag_diffusion(nx, ny, dx, dy)
        b = np.zeros((ny + 2, nx + 2)); b[1:-1, 1:-1] = 1.0 / ((nx + 1) * (ny + 1))
        s = oracle.Solver(so, relax=relax, maxiter=30, tol=1e-10)
        x, h = s.solve(b)
        r = oracle.residual(np.ascontiguousarray(so), x, b)
        assert np.linalg.norm(r) < 1e-8


# ------------------------------------------------------------------------- 3D
@pytest.mark.parametrize("n", [7, 8, 9])
def test_3d_galerkin_and_restriction_are_ptap_and_pt(oracle, n):
    rng = np.random.default_rng(n)
    k = np.exp(rng.normal(size=(n + 1,) * 3))
    so = G.fe3_hetero(k)
    nc = (n - 1) // 2 + 1
    ci = oracle.setup_interp3(so, nc, nc, nc)
    soc = oracle.galerkin3(so, ci)
    A = G.stencil3_to_csr(so).toarray()
    Pm = np.zeros((n ** 3, nc ** 3))
    for kc in range(nc):
        for jc in range(nc):
            for ic in range(nc):
                xc = np.zeros((nc + 2,) * 3)
                xc[kc + 1, jc + 1, ic + 1] = 1
                xf = np.zeros((n + 2,) * 3)
                oracle.interp_add3(ci, xc, np.zeros_like(xf), so, xf)
                Pm[:, (kc * nc + jc) * nc + ic] = xf[1:-1, 1:-1, 1:-1].ravel()
    Ac = Pm.T @ A @ Pm
    assert np.abs(Ac - G.stencil3_to_csr(soc).toarray()).max() <= 1e-14 * np.abs(Ac).max()
    r = np.zeros((n + 2,) * 3)
    r[1:-1, 1:-1, 1:-1] = rng.random((n, n, n))
    bc = oracle.restrict3(ci, r)
    np.testing.assert_allclose(bc[1:-1, 1:-1, 1:-1].ravel(), Pm.T @ r[1:-1, 1:-1, 1:-1].ravel(), rtol=1e-13, atol=1e-14)
    # interpolation reproduces constants away from the boundary on a constant-coefficient operator
    soc1 = G.fe3_hetero(np.ones((n + 1,) * 3))
    ci1 = oracle.setup_interp3(soc1, nc, nc, nc)
    xc = np.zeros((nc + 2,) * 3)
    xc[1:-1, 1:-1, 1:-1] = 1.0
    xf = np.zeros((n + 2,) * 3)
    oracle.interp_add3(ci1, xc, np.zeros_like(xf), soc1, xf)
    assert abs(xf[n // 2, n // 2, n // 2] - 1.0) < 1e-12


def test_3d_residual_matches_assembled_matrix(oracle):
    n = 9
    rng = np.random.default_rng(3)
    so = G.fe3_hetero(np.exp(rng.normal(size=(n + 1,) * 3)))
    A = G.stencil3_to_csr(so)
    assert abs(A - A.T).max() == 0
    x = np.zeros((n + 2,) * 3); x[1:-1, 1:-1, 1:-1] = rng.random((n, n, n))
    b = np.zeros_like(x); b[1:-1, 1:-1, 1:-1] = rng.random((n, n, n))
    r = oracle.residual3(so, x, b)
    np.testing.assert_allclose(r[1:-1, 1:-1, 1:-1].ravel(), b[1:-1, 1:-1, 1:-1].ravel() - A @ x[1:-1, 1:-1, 1:-1].ravel(),
                               atol=1e-14)


def test_3d_boxmg_converges(oracle):
    n = 15
    rng = np.random.default_rng(4)
    so = G.fe3_hetero(np.exp(1.5 * rng.normal(size=(n + 1,) * 3)))
    b = np.zeros((n + 2,) * 3); b[1:-1, 1:-1, 1:-1] = rng.uniform(-1, 1, (n, n, n)) / (n + 1) ** 3
    s = oracle.Solver3(so, maxiter=20, tol=1e-10)
    x, h = s.solve(b)
    assert h[-1] < 1e-10 and len(h) <= 12
    assert oracle.num_levels(15, 15, 3) == 3


def _block_gs_planes(A, nx, ny, nz, direction, x, b, updown):
    """Red-black block Gauss-Seidel over planes with exact plane solves (dense)."""
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    if direction == "xy":
        planes = [idx[k].ravel() for k in range(nz)]
    elif direction == "xz":
        planes = [idx[:, j, :].ravel() for j in range(ny)]
    else:
        planes = [idx[:, :, i].ravel() for i in range(nx)]
    n = len(planes)
    order = [range(0, n, 2), range(1, n, 2)]
    if updown == 1:
        order = order[::-1]
    xv = x[1:-1, 1:-1, 1:-1].ravel().copy()
    bv = b[1:-1, 1:-1, 1:-1].ravel()
    for rng in order:
        for p in rng:
            ip = planes[p]
            rhs = bv[ip] - A[ip] @ xv + A[np.ix_(ip, ip)] @ xv[ip]
            xv[ip] = np.linalg.solve(A[np.ix_(ip, ip)], rhs)
    out = x.copy()
    out[1:-1, 1:-1, 1:-1] = xv.reshape(nz, ny, nx)
    return out


@pytest.mark.parametrize("direction", ["xy", "xz", "yz"])
def test_3d_plane_relaxation_is_block_gauss_seidel(oracle, direction):
    # 4 x 4 planes have a one-level 2D hierarchy, so each plane solve is the exact
    # banded Cholesky: a plane sweep is then red-black block Gauss-Seidel
    nx, ny, nz = 4, 4, 4
    rng = np.random.default_rng(21)
    so = G.fe3_hetero(np.exp(rng.normal(size=(nz + 1, ny + 1, nx + 1))))
    A = G.stencil3_to_csr(so).toarray()
    s = oracle.Solver3(so, relax="plane-xyz", min_coarse=2)
    assert s.nlevels == 2
    for updown in (0, 1):
        x = np.zeros((nz + 2, ny + 2, nx + 2)); x[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
        b = np.zeros_like(x); b[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
        ref = _block_gs_planes(A, nx, ny, nz, direction, x, b, updown)
        got = s.relax_planes(0, direction, x.copy(), b, updown)
        np.testing.assert_allclose(got[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1], rtol=1e-11, atol=1e-13)


def test_3d_plane_operators_are_the_in_plane_couplings(oracle):
    nx, ny, nz = 5, 6, 7
    rng = np.random.default_rng(22)
    so = G.fe3_hetero(np.exp(rng.normal(size=(nz + 1, ny + 1, nx + 1))))
    A = G.stencil3_to_csr(so).toarray()
    s = oracle.Solver3(so, relax="plane-xyz", num_levels=2)
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    for direction, ipl in (("xy", 3), ("xz", 2), ("yz", 4)):
        so2 = s.plane_op(0, direction, ipl)
        ip = (idx[ipl - 1] if direction == "xy" else idx[:, ipl - 1, :] if direction == "xz" else idx[:, :, ipl - 1]).ravel()
        A2 = G.stencil_to_csr(so2).toarray()
        np.testing.assert_array_equal(A2, A[np.ix_(ip, ip)])


def test_3d_plane_boxmg_converges(oracle):
    n = 15
    rng = np.random.default_rng(23)
    so = G.fe3_hetero(np.exp(1.5 * rng.normal(size=(n + 1,) * 3)))
    b = np.zeros((n + 2,) * 3); b[1:-1, 1:-1, 1:-1] = rng.uniform(-1, 1, (n, n, n)) / (n + 1) ** 3
    _, hp = oracle.Solver3(so, maxiter=12, tol=1e-10, relax="plane-xyz").solve(b)
    _, h0 = oracle.Solver3(so, maxiter=12, tol=1e-10).solve(b)
    assert hp[-1] < 1e-10 and len(hp) <= len(h0)


# ----------------------------------------------------------- 3D seven-point
def _gs7_dense(A, x, b, updown):
    """Red-black Gauss-Seidel on the assembled matrix: colour pts holds the points
    with I+J+K+pts even in the reference's 1-based indices (I = numpy index + 1
    with the ghost at 0), colour 0 first going up."""
    nz, ny, nx = x.shape[0] - 2, x.shape[1] - 2, x.shape[2] - 2
    K, J, I = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    par = ((I + J + K + 3) % 2).ravel()
    xv = x[1:-1, 1:-1, 1:-1].ravel().copy()
    bv = b[1:-1, 1:-1, 1:-1].ravel()
    for pts in ((0, 1) if updown == 1 else (1, 0)):
        idx = np.nonzero((par + pts) % 2 == 0)[0]
        d = A.diagonal()[idx]
        xv[idx] = (bv[idx] - (A[idx] @ xv - d * xv[idx])) / d
    out = x.copy()
    out[1:-1, 1:-1, 1:-1] = xv.reshape(nz, ny, nx)
    return out


def _op7(nx, ny, nz, seed, sigma=1.0):
    rng = np.random.default_rng(seed)
    return G.fd3_hetero(np.exp(sigma * rng.normal(size=(nz + 2, ny + 2, nx + 2))))


@pytest.mark.parametrize("n", [(7, 6, 5), (8, 9, 10)])
def test_3d_seven_point_residual_and_gs_match_assembled_matrix(oracle, n):
    nx, ny, nz = n
    so = _op7(nx, ny, nz, seed=31)
    A = G.stencil3_to_csr(so)
    assert abs(A - A.T).max() == 0
    rng = np.random.default_rng(32)
    x = np.zeros((nz + 2, ny + 2, nx + 2)); x[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
    b = np.zeros_like(x); b[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
    r = oracle.residual3(so, x, b)
    np.testing.assert_allclose(r[1:-1, 1:-1, 1:-1].ravel(), b[1:-1, 1:-1, 1:-1].ravel() - A @ x[1:-1, 1:-1, 1:-1].ravel(),
                               atol=1e-14)
    sor = oracle.setup_recip3(so)
    for updown in (0, 1):
        got = oracle.relax_gs3(so, x.copy(), b, sor, updown)
        np.testing.assert_allclose(got, _gs7_dense(A, x, b, updown), rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("n", [7, 8, 9])
def test_3d_seven_point_interpolation_and_galerkin(oracle, n):
    """Edge weights equal the 27-point branch's on the zero-padded operator (the
    27-point sums reduce to the seven-point ones term by term); the Galerkin
    operator is P^T A P; constants are reproduced away from the boundary."""
    so = _op7(n, n, n, seed=n, sigma=1.2)
    nc = (n - 1) // 2 + 1
    ci = oracle.setup_interp3(so, nc, nc, nc)
    ci27 = oracle.setup_interp3(G.seven_to_27(so), nc, nc, nc)
    for l in range(6):  # lxyl lxyr lxya lxyb lxza lxzb
        np.testing.assert_array_equal(ci[l], ci27[l])
    soc = oracle.galerkin3(so, ci)
    A = G.stencil3_to_csr(so).toarray()
    Pm = np.zeros((n ** 3, nc ** 3))
    for kc in range(nc):
        for jc in range(nc):
            for ic in range(nc):
                xc = np.zeros((nc + 2,) * 3)
                xc[kc + 1, jc + 1, ic + 1] = 1
                xf = np.zeros((n + 2,) * 3)
                oracle.interp_add3(ci, xc, np.zeros_like(xf), so, xf)
                Pm[:, (kc * nc + jc) * nc + ic] = xf[1:-1, 1:-1, 1:-1].ravel()
    Ac = Pm.T @ A @ Pm
    assert np.abs(Ac - G.stencil3_to_csr(soc).toarray()).max() <= 1e-14 * np.abs(Ac).max()
    so1 = G.poisson3(n, n, n)
    ci1 = oracle.setup_interp3(so1, nc, nc, nc)
    xc = np.zeros((nc + 2,) * 3); xc[1:-1, 1:-1, 1:-1] = 1.0
    xf = np.zeros((n + 2,) * 3)
    oracle.interp_add3(ci1, xc, np.zeros_like(xf), so1, xf)
    assert abs(xf[n // 2, n // 2, n // 2] - 1.0) < 1e-12


def test_3d_seven_point_poisson_known_answer(oracle):
    """test/3d/test_poisson.cc:73-104 (SerialPoisson3.Isotropic) at n = 39 instead
    of 200: the default solve ends with ||r||_2 < 1e-8, and the error against
    sin(2 pi x) sin(2 pi y) sin(2 pi z) is the O(h^2) discretisation error
    (below 1e-4 at n = 200; scaled by (201/40)^2 here)."""
    n = 39
    so = G.poisson3(n, n, n)
    b = G.poisson3_rhs_sin2pi(n, n, n)
    s = oracle.Solver3(so)
    x, h = s.solve(b)
    r = oracle.residual3(so, x, b)
    assert oracle.l2norm3(r) < 1e-8
    err = np.abs(x - G.poisson3_exact_sin2pi(n, n, n))[1:-1, 1:-1, 1:-1].max()
    assert err < 1e-4 * (201 / 40) ** 2
    assert h[-1] < 1e-8 and len(h) <= 10


@pytest.mark.parametrize("direction", ["xy", "xz", "yz"])
def test_3d_seven_point_plane_relaxation_is_block_gauss_seidel(oracle, direction):
    nx, ny, nz = 4, 4, 4
    so = _op7(nx, ny, nz, seed=33)
    A = G.stencil3_to_csr(so).toarray()
    s = oracle.Solver3(so, relax="plane-xyz", min_coarse=2)
    assert s.nlevels == 2
    rng = np.random.default_rng(34)
    for updown in (0, 1):
        x = np.zeros((nz + 2, ny + 2, nx + 2)); x[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
        b = np.zeros_like(x); b[1:-1, 1:-1, 1:-1] = rng.random((nz, ny, nx))
        ref = _block_gs_planes(A, nx, ny, nz, direction, x, b, updown)
        got = s.relax_planes(0, direction, x.copy(), b, updown)
        np.testing.assert_allclose(got[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1], rtol=1e-11, atol=1e-13)
    # each plane's five-point operator is the in-plane block of A
    s2 = oracle.Solver3(_op7(5, 6, 7, seed=35), relax="plane-xyz", num_levels=2)
    A2full = G.stencil3_to_csr(_op7(5, 6, 7, seed=35)).toarray()
    idx = np.arange(5 * 6 * 7).reshape(7, 6, 5)
    ipl = 2
    so2 = s2.plane_op(0, direction, ipl)
    ip = (idx[ipl - 1] if direction == "xy" else idx[:, ipl - 1, :] if direction == "xz" else idx[:, :, ipl - 1]).ravel()
    assert not so2[3:].any()
    np.testing.assert_array_equal(G.stencil_to_csr(np.ascontiguousarray(so2[:3])).toarray(), A2full[np.ix_(ip, ip)])


def test_3d_seven_point_boxmg_converges_both_smoothers(oracle):
    n = 15
    so = _op7(n, n, n, seed=36, sigma=1.5)
    rng = np.random.default_rng(37)
    b = np.zeros((n + 2,) * 3); b[1:-1, 1:-1, 1:-1] = rng.uniform(-1, 1, (n, n, n)) / (n + 1) ** 3
    _, h0 = oracle.Solver3(so, maxiter=20, tol=1e-10).solve(b)
    _, hp = oracle.Solver3(so, maxiter=20, tol=1e-10, relax="plane-xyz").solve(b)
    assert h0[-1] < 1e-10 and hp[-1] < 1e-10 and len(hp) <= len(h0)


_THREAD_PROBE = r"""
import hashlib, sys
sys.path.insert(0, sys.argv[1])
from oracle import oracle
from cedar_b200 import problems as P
so, b = P.hetero_diffusion(767, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
out = [str(oracle.num_threads())]
for relax in ("line-xy", "point"):
    x, h = oracle.Solver(so, relax=relax, maxiter=2, tol=0).solve(b)
    out.append(hashlib.sha256(x.tobytes()).hexdigest())
print(" ".join(out))
"""


def test_oracle_threads_do_not_change_results(oracle):
    """The 2D cycle kernels split rows / lines of one colour over host threads
    (ORACLE_THREADS); every element gets the same operations, so one thread
    and four give the same bits (767^2 is above the threading threshold)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for t in ("1", "4"):
        p = subprocess.run([sys.executable, "-c", _THREAD_PROBE, root], env=dict(os.environ, ORACLE_THREADS=t),
                           capture_output=True, text=True, check=True, timeout=300)
        res[t] = p.stdout.split()
    assert res["1"][0] == "1" and res["4"][0] == "4"
    assert res["1"][1:] == res["4"][1:]


# ----------------------------------------------------------------- F-cycle
def test_fcycle_two_levels_is_vcycle_from_interpolated_coarse_solve(oracle):
    """cycle::fcycle (include/cedar/cycle/fcycle.h:49-83) on two levels: restrict
    b, solve the coarse system exactly, x = P x_c (zero residual term), then one
    V-cycle from that x.  Restated here with the oracle's own kernels and
    compared bit for bit; the incoming x does not matter."""
    n = 31
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
    so = np.ascontiguousarray(so)
    sf = oracle.Solver(so, relax="line-xy", num_levels=2, maxiter=1, tol=0, cycle="f")
    x_f, h_f = sf.solve(b, x=np.random.default_rng(0).random(b.shape))
    ci = sf.level_array(1, "ci")
    soc = sf.level_array(1, "so")
    bc = oracle.restrict(ci, b)
    abd, info = oracle.setup_cg(soc)
    assert info == 0
    xc = oracle.solve_cg(abd, bc)
    x0 = oracle.interp_add(ci, xc, np.zeros_like(b), so, np.zeros_like(b))
    sv = oracle.Solver(so, relax="line-xy", num_levels=2, maxiter=1, tol=0)
    x_v = sv.vcycle(x0.copy(), b)
    np.testing.assert_array_equal(x_f, x_v)


def test_fcycle_solve_repeats_the_same_iterate(oracle):
    """The reference's solve loop hands the F-cycle the current x, which
    fmg_cycle discards: every iteration gives the same x and residual."""
    n = 63
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
    x, h = oracle.Solver(so, relax="line-xy", maxiter=4, tol=0, cycle="f").solve(b)
    assert len(h) == 4 and np.all(h == h[0]) and h[0] < 0.5


def test_fcycle3_two_levels_is_vcycle_from_interpolated_coarse_solve(oracle):
    """The 3D F-cycle (the same cycle::fcycle template, include/cedar/cycle/fcycle.h:49-83)
    on two levels: restrict b, solve the coarse system exactly, x = P x_c with a
    zero residual term, then one V-cycle from that x; the oracle's 3D kernels
    composed here give the same bits, whatever the incoming x."""
    from cedar_b200 import gallery as G
    from cedar_b200 import problems as P3
    n = 7
    k = P3.hetero3_coefficients(n, sigma=1.0, n_incl=2, contrast=10.0)
    so = np.ascontiguousarray(G.fe3_hetero(k))
    b = P3.hetero3_rhs(n)
    sf = oracle.Solver3(so, num_levels=2, maxiter=1, tol=0, cycle="f")
    x_f, _ = sf.solve(b, x=np.random.default_rng(0).random(b.shape))
    ci = sf.level_array(1, "ci")
    soc = sf.level_array(1, "so")
    abd, info = oracle.setup_cg3(soc)
    assert info == 0
    xc = oracle.solve_cg3(abd, oracle.restrict3(ci, b))
    x0 = oracle.interp_add3(ci, xc, np.zeros_like(b), so, np.zeros_like(b))
    x_v = oracle.Solver3(so, num_levels=2, maxiter=1, tol=0).vcycle(x0.copy(), b)
    np.testing.assert_array_equal(x_f, x_v)
