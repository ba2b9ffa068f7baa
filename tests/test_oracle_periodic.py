"""CPU checks of the oracle's periodic branches (oracle/cdr2_periodic.c).

The reference holds no periodic golden values, so the restatement is pinned by
identities on the wrapped grid (the matrix assembled with the periodic
couplings, ghost lines holding copies of the opposite interior lines):
Galerkin operator = P^T A P with P taken from the periodic interpolation,
restriction = P^T, one Gauss-Seidel sweep = the reference's sequential sweep
written directly on the wrapped matrix, the dense coarsest factor = the
Cholesky factor of that matrix; and by the reference's periodic example
(examples/basic-2d-ser/periodic.cc), whose solve converges to the
discretisation error of the exact solution.
"""
import numpy as np
import pytest

from cedar_b200 import gallery as G

PERS = [(True, False), (False, True), (True, True)]


def wrap_copy(x, per):
    if per[0]:
        x[..., :, 0] = x[..., :, -2]
        x[..., :, -1] = x[..., :, 1]
    if per[1]:
        x[..., 0, :] = x[..., -2, :]
        x[..., -1, :] = x[..., 1, :]
    return x


def assemble(so, per):
    """Dense matrix of a stencil on the wrapped grid."""
    ns, JJ, II = so.shape
    ny, nx = JJ - 2, II - 2
    A = np.zeros((nx * ny, nx * ny))

    def idx(i, j):
        if per[0]:
            i = nx if i == 0 else (1 if i == nx + 1 else i)
        if per[1]:
            j = ny if j == 0 else (1 if j == ny + 1 else j)
        return (j - 1) * nx + (i - 1) if 1 <= i <= nx and 1 <= j <= ny else None

    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            p = idx(i, j)
            A[p, p] += so[0, j, i]
            nb = [((i - 1, j), so[1, j, i]), ((i + 1, j), so[1, j, i + 1]), ((i, j - 1), so[2, j, i]),
                  ((i, j + 1), so[2, j + 1, i])]
            if ns == 5:
                nb += [((i - 1, j - 1), so[3, j, i]), ((i + 1, j + 1), so[3, j + 1, i + 1]),
                       ((i - 1, j + 1), so[4, j + 1, i]), ((i + 1, j - 1), so[4, j, i + 1])]
            for (a, c), v in nb:
                q = idx(a, c)
                if q is not None:
                    A[p, q] -= v
    return A


def periodic_op(n, ns, per, seed):
    """A definite heterogeneous periodic operator (wrap couplings set, ghosts copied)."""
    rng = np.random.default_rng(seed)
    if ns == 3:
        so, _, _ = G.periodic_poisson(n, n, per)
        so[1:, 1:-1, 1:-1] *= 1 + 0.3 * rng.random((2, n, n))
    else:
        k = np.exp(rng.normal(size=(n + 1, n + 1)))
        so = G.fe_hetero(k, k)
        if per[0]:
            so[1:, 1:-1, 1] = so[1:, 1:-1, 2]
        if per[1]:
            so[2:, 1, 1:-1] = so[2:, 2, 1:-1]
            so[1, 1, 1:-1] = so[1, 2, 1:-1]
    for pl in range(1, ns):
        wrap_copy(so[pl], per)
    # diagonal = wrapped row sum of the couplings + a shift: diagonally dominant, so definite
    so[0] = 0.0
    so[0, 1:-1, 1:-1] = -assemble(so, per).sum(axis=1).reshape(n, n) + 0.05
    wrap_copy(so[0], per)
    return np.ascontiguousarray(so)


def prolongation(oracle, ci, so, n, nxc, per, ipn):
    Pm = np.zeros((n * n, nxc * nxc))
    for jc in range(nxc):
        for ic in range(nxc):
            xc = np.zeros((nxc + 2, nxc + 2))
            xc[jc + 1, ic + 1] = 1.0
            wrap_copy(xc, per)
            xf = np.zeros((n + 2, n + 2))
            oracle.interp_add_per(ci, xc, np.zeros_like(xf), so, xf, ipn)
            Pm[:, jc * nxc + ic] = xf[1:-1, 1:-1].ravel()
    return Pm


@pytest.mark.parametrize("per", PERS)
@pytest.mark.parametrize("n,ns", [(16, 3), (16, 5), (20, 5), (24, 3)])
def test_periodic_galerkin_is_ptap_and_restriction_is_pt(oracle, per, n, ns):
    so = periodic_op(n, ns, per, seed=n + ns)
    ipn = oracle.bc_code(per)
    nxc = (n - 1) // 2 + 1
    ci = oracle.setup_interp_per(so, nxc, nxc, ipn)
    soc = oracle.galerkin_per(so, ci, ipn)
    A = assemble(so, per)
    Pm = prolongation(oracle, ci, so, n, nxc, per, ipn)
    Ac = Pm.T @ A @ Pm
    assert np.abs(Ac - assemble(soc, per)).max() <= 1e-13 * np.abs(Ac).max()
    # the coarse operator's ghost lines hold copies of the opposite interior lines
    for pl in range(5):
        np.testing.assert_array_equal(soc[pl], wrap_copy(soc[pl].copy(), per))
    # restriction = P^T on the wrapped grid
    rng = np.random.default_rng(7)
    r = np.zeros((n + 2, n + 2))
    r[1:-1, 1:-1] = rng.standard_normal((n, n))
    bc = oracle.restrict_per(ci, wrap_copy(r.copy(), per), ipn)
    np.testing.assert_allclose(bc[1:-1, 1:-1].ravel(), Pm.T @ r[1:-1, 1:-1].ravel(), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("per", PERS)
@pytest.mark.parametrize("n,ns", [(19, 3), (21, 5), (37, 5)])
def test_odd_periodic_galerkin_off_the_seam(oracle, per, n, ns):
    """Odd periodic sizes: the last and first coarse points are fine
    neighbours across the seam, yet the reference's product is the definite
    loop plus ghost copies (src/2d/ftn/BMG2_SymStd_SETUP_ITLI_ex.f90:216-247),
    which treats the fine ghost line (a copy of a coarse point) as a fine
    point between them.  So the coarse operator equals P^T A P everywhere
    except in the couplings of the two coarse lines at the seam, and differs
    there -- the reference's own behaviour, restated."""
    so = periodic_op(n, ns, per, seed=n)
    ipn = oracle.bc_code(per)
    nxc = (n - 1) // 2 + 1
    ci = oracle.setup_interp_per(so, nxc, nxc, ipn)
    soc = oracle.galerkin_per(so, ci, ipn)
    Pm = prolongation(oracle, ci, so, n, nxc, per, ipn)
    Ac = Pm.T @ assemble(so, per) @ Pm
    G = assemble(soc, per)
    ic, jc = np.meshgrid(np.arange(1, nxc + 1), np.arange(1, nxc + 1))
    seam = np.zeros((nxc, nxc), bool)
    if per[0]:
        seam |= (ic == 1) | (ic == nxc)
    if per[1]:
        seam |= (jc == 1) | (jc == nxc)
    off = ~seam.ravel()
    blk = np.ix_(off, off)
    assert np.abs(Ac[blk] - G[blk]).max() <= 1e-13 * np.abs(Ac).max()
    assert np.abs(Ac - G).max() > 1e-2 * np.abs(Ac).max()


@pytest.mark.parametrize("per", PERS)
@pytest.mark.parametrize("ns", [3, 5])
def test_periodic_gauss_seidel_sweep(oracle, per, ns):
    """One sweep of the periodic branch = the reference's sequential loops
    written on the wrapped matrix (the ghost copies it refreshes after each
    row are what the next points read): compared point by point."""
    n = 12
    so = periodic_op(n, ns, per, seed=ns)
    ipn = oracle.bc_code(per)
    sor = oracle.setup_recip(so)
    rng = np.random.default_rng(2)
    b = np.zeros((n + 2, n + 2))
    b[1:-1, 1:-1] = rng.standard_normal((n, n))
    x0 = wrap_copy(np.pad(rng.standard_normal((n, n)), 1), per)
    for updown in (0, 1):
        x = oracle.relax_gs_per(so, x0.copy(), b, sor, updown, ipn)
        # sequential restatement in Python (the loop order of relax_GS.f90:139-226)
        q = x0.copy()
        I1, J1 = n, n
        ls = (2, 3) if updown == 0 else (3, 2)

        def upd(I, J):
            i, j = I - 1, J - 1  # 0-based array indices
            acc = b[j, i] + so[1, j, i] * q[j, i - 1] + so[1, j, i + 1] * q[j, i + 1] + so[2, j, i] * q[j - 1, i] \
                + so[2, j + 1, i] * q[j + 1, i]
            if ns == 5:
                acc = acc + so[3, j, i] * q[j - 1, i - 1] + so[4, j, i + 1] * q[j - 1, i + 1] \
                    + so[4, j + 1, i] * q[j + 1, i - 1] + so[3, j + 1, i + 1] * q[j + 1, i + 1]
            q[j, i] = acc * sor[1, j, i]

        def ghost_x(J):
            if per[0]:
                q[J - 1, 0] = q[J - 1, I1]
                q[J - 1, I1 + 1] = q[J - 1, 1]

        if ns == 5:
            for JBEG in ls:
                for J in range(JBEG, J1 + 2, 2):
                    for IBEG in ls:
                        for I in range(IBEG, I1 + 2, 2):
                            upd(I, J)
                        ghost_x(J)
        else:
            for JO in ls:
                for J in range(2, J1 + 2):
                    for I in range((J + JO) % 2 + 2, I1 + 2, 2):
                        upd(I, J)
                    ghost_x(J)
        if per[1]:
            q[0, :] = q[J1, :]
            q[J1 + 1, :] = q[1, :]
        np.testing.assert_allclose(x, q, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("per", PERS)
@pytest.mark.parametrize("ns", [3, 5])
def test_periodic_coarse_factor_and_solve(oracle, per, ns):
    """The dense coarsest factor is the Cholesky factor of the wrapped matrix
    (DPOTF2 order, equal to numpy to rounding); the solve returns the
    zero-mean shift of A^{-1} b with its ghost lines filled."""
    n = 6
    so = periodic_op(n, ns, per, seed=11 + ns)
    ipn = oracle.bc_code(per)
    abd, info = oracle.setup_cg_per(so, ipn)
    assert info == 0
    A = assemble(so, per)
    U = np.triu(abd.T)  # the factor is column-major
    np.testing.assert_allclose(U, np.linalg.cholesky(A).T, rtol=1e-12, atol=1e-12)
    rng = np.random.default_rng(9)
    b = np.zeros((n + 2, n + 2))
    b[1:-1, 1:-1] = rng.standard_normal((n, n))
    x = oracle.solve_cg_per(abd, b, ipn)
    xs = np.linalg.solve(A, b[1:-1, 1:-1].ravel())
    np.testing.assert_allclose(x[1:-1, 1:-1].ravel(), xs - xs.mean(), rtol=1e-11, atol=1e-12)
    np.testing.assert_array_equal(x, wrap_copy(x.copy(), per))


def transpose_op(so):
    """The operator of the transposed grid (x <-> y): W and S planes swap, SW and NW keep their kind."""
    planes = [0, 2, 1] if so.shape[0] == 3 else [0, 2, 1, 3, 4]
    return np.ascontiguousarray(np.stack([so[p].T for p in planes]))


@pytest.mark.parametrize("ns", [3, 5])
def test_periodic_x_and_y_branches_are_transposes(oracle, ns):
    """The x- and y-periodic branches of the interpolation, Galerkin product,
    restriction and interpolation are separate code in the reference; on the
    transposed problem they must give the transposed results (LL <-> LB,
    LR <-> LA, LNW <-> LSE)."""
    n = 16
    sox = periodic_op(n, ns, (True, False), seed=5)
    soy = transpose_op(sox)
    ipx, ipy = oracle.bc_code((True, False)), oracle.bc_code((False, True))
    nxc = (n - 1) // 2 + 1
    cix = oracle.setup_interp_per(sox, nxc, nxc, ipx)
    ciy = oracle.setup_interp_per(soy, nxc, nxc, ipy)
    perm = [3, 2, 1, 0, 4, 7, 6, 5]
    np.testing.assert_allclose(ciy, np.stack([cix[p].T for p in perm]), rtol=1e-14, atol=1e-15)
    socx = oracle.galerkin_per(sox, cix, ipx)
    socy = oracle.galerkin_per(soy, ciy, ipy)
    np.testing.assert_allclose(socy, transpose_op(socx), rtol=1e-13, atol=1e-13)
    rng = np.random.default_rng(3)
    r = np.pad(rng.standard_normal((n, n)), 1)
    bx = oracle.restrict_per(cix, wrap_copy(r.copy(), (True, False)), ipx)
    by = oracle.restrict_per(ciy, wrap_copy(np.ascontiguousarray(r.T), (False, True)), ipy)
    np.testing.assert_allclose(by, bx.T, rtol=1e-14, atol=1e-14)
    xc = np.pad(rng.standard_normal((nxc, nxc)), 1)
    z = np.zeros((n + 2, n + 2))
    fx = oracle.interp_add_per(cix, wrap_copy(xc.copy(), (True, False)), z.copy(), sox, z.copy(), ipx)
    fy = oracle.interp_add_per(ciy, wrap_copy(np.ascontiguousarray(xc.T), (False, True)), z.copy(), soy, z.copy(),
                               ipy)
    np.testing.assert_allclose(fy, fx.T, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("per", [(True, False), (False, True)])
def test_periodic_example_converges_to_the_discretisation_error(oracle, per):
    """The reference's periodic example (5-point Poisson, V(1,1) point
    relaxation, 1e-10; examples/basic-2d-ser/periodic-config.json) at 64^2
    and 128^2, and the transposed problem.  x-periodic: converges in the
    example's ten cycles (contraction about 0.09).  y-periodic: the reference's
    sweep copies the y ghost rows only after both colours
    (src/2d/ftn/BMG2_SymStd_relax_GS.f90:199-225), so the second colour reads
    the first colour's stale ghost rows and the cycle contracts by about 0.6
    once the smooth error is gone; ten cycles still reach 1e-7.  In both the
    error against sin(2 pi x) sin(2 pi y) falls by 4 with h."""
    errs = []
    for n in (64, 128):
        so, b, ex = G.periodic_poisson(n, n, per)
        s = oracle.Solver(so, relax="point", nrelax_pre=1, nrelax_post=1, maxiter=10, tol=1e-10, periodic=per)
        x, h = s.solve(b)
        assert np.all(np.diff(h) < 0)
        if per[0]:
            assert h[-1] < 1e-10 and len(h) <= 10
        else:
            assert len(h) == 10 and h[-1] < 1e-7 and 0.45 < h[-1] / h[-2] < 0.75
        errs.append(np.abs(x[1:-1, 1:-1] - ex[1:-1, 1:-1]).max())
    assert 3.5 < errs[0] / errs[1] < 4.5
