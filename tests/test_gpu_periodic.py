"""Periodic boundary conditions on the GPU against the oracle (grid.periodic).

Every periodic kernel keeps the reference's operand order, so the hierarchy
(interpolation weights, Galerkin operators with their ghost lines) and the
iterates are bit-identical to the oracle's; the residual norms, reduced in
parallel, agree to rounding.  Cases: x-, y- and xy-periodic; five- and
nine-point operators; even and odd grids (the odd ones take the reference's
wrapped column walk of the interpolation setup) and a non-square one; V and F
cycles; the reference's periodic example (examples/basic-2d-ser/periodic.cc
with periodic-config.json)."""
import numpy as np
import pytest

from cedar_b200 import gallery as G
from cedar_b200.config import Config
from tests.test_oracle_periodic import assemble, wrap_copy

pytestmark = pytest.mark.gpu
PERS = {"x": (True, False), "y": (False, True), "xy": (True, True)}


def gpu(so, per, **kw):
    from cedar_b200.solver import Solver2D
    conf = {"solver": {"relaxation": "point", "max-iter": kw.get("maxiter", 4), "tol": kw.get("tol", 0.0),
                       "cycle": {"nrelax-pre": kw.get("pre", 2), "nrelax-post": kw.get("post", 1),
                                 "type": kw.get("cycle", "v")}},
            "grid": {"periodic": [per[0], per[1], False]},
            "gpu": {"graph": kw.get("graph", True)}}
    return Solver2D(so, Config(conf))


def problem(nx, ny, ns, per, seed):
    """A random definite periodic operator (positive couplings copied into the
    ghost lines of the periodic directions, diagonal = wrapped row sum + 0.05)
    and a random right-hand side with its ghost copies."""
    rng = np.random.default_rng(seed)
    so = np.zeros((ns, ny + 2, nx + 2))
    so[1:3, 1:-1, 1:-1] = 0.5 + rng.random((2, ny, nx))
    if ns == 5:
        so[3:, 1:-1, 1:-1] = 0.25 * rng.random((2, ny, nx))
    for pl in range(1, ns):
        wrap_copy(so[pl], per)
    so[0, 1:-1, 1:-1] = -assemble(so, per).sum(axis=1).reshape(ny, nx) + 0.05
    wrap_copy(so[0], per)
    b = np.zeros((ny + 2, nx + 2))
    b[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    return np.ascontiguousarray(so), wrap_copy(b, per)


CASES = [("x", 3, 64, 64), ("y", 3, 64, 64), ("xy", 3, 64, 64), ("x", 5, 75, 75), ("y", 5, 75, 75),
         ("xy", 5, 75, 75), ("xy", 3, 99, 99), ("x", 5, 96, 41), ("y", 3, 41, 96)]


@pytest.mark.parametrize("pk,ns,nx,ny", CASES)
def test_periodic_hierarchy_and_iterates_match_oracle(oracle, pk, ns, nx, ny):
    per = PERS[pk]
    so, b = problem(nx, ny, ns, per, seed=nx + ns)
    s = gpu(so, per, maxiter=4)
    o = oracle.Solver(so, relax="point", maxiter=4, tol=0.0, periodic=per)
    assert o.info() == (0, 0)
    assert s.nlevels == o.nlevels
    for l in range(s.nlevels):
        np.testing.assert_array_equal(s.level_array(l, "so"), o.level_array(l, "so"), err_msg="so level %d" % l)
        if l > 0:
            np.testing.assert_array_equal(s.level_array(l, "ci"), o.level_array(l, "ci"), err_msg="ci level %d" % l)
    x = s.solve(b)
    xo, ho = o.solve(b)
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_allclose(s.history, ho, rtol=1e-12)


@pytest.mark.parametrize("pk", ["x", "xy"])
def test_periodic_fcycle_matches_oracle(oracle, pk):
    per = PERS[pk]
    so, b = problem(63, 63, 5, per, seed=7)
    s = gpu(so, per, maxiter=3, cycle="f")
    o = oracle.Solver(so, relax="point", maxiter=3, tol=0.0, periodic=per, cycle="f")
    x = s.solve(b)
    xo, ho = o.solve(b)
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_allclose(s.history, ho, rtol=1e-12)


@pytest.mark.parametrize("graph", [True, False])
def test_reference_periodic_example(oracle, graph):
    """examples/basic-2d-ser/periodic.cc with its config: 300^2 Poisson, x
    periodic, V(1,1) point relaxation, tolerance 1e-10, at most 10 cycles.
    The hierarchy passes odd periodic sizes (75, 19, 5), where the
    reference's coarse operator is not Galerkin at the seam, so the ten
    cycles end near 5e-6 rather than at the tolerance, as the oracle's do.
    Same iterates as the oracle; the solution is within 1e-4 of
    sin(2 pi x) sin(2 pi y)."""
    per = (True, False)
    so, b, ex = G.periodic_poisson(300, 300, per)
    s = gpu(so, per, maxiter=10, tol=1e-10, pre=1, post=1, graph=graph)
    o = oracle.Solver(so, relax="point", nrelax_pre=1, nrelax_post=1, maxiter=10, tol=1e-10, periodic=per)
    x = s.solve(b)
    xo, ho = o.solve(b)
    assert s.iters == len(ho) == 10 and ho[-1] < 1e-5
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_allclose(s.history, ho, rtol=1e-12)
    assert np.abs(x[1:-1, 1:-1] - ex[1:-1, 1:-1]).max() < 1e-4


def test_periodic_unsupported_options_are_refused():
    from cedar_b200 import _lib
    from cedar_b200.solver import Solver2D
    so, _ = problem(32, 32, 3, (True, False), seed=1)
    for extra in ({"solver": {"relaxation": "line-x"}}, {"gpu": {"precision": "fp32-ir"}},
                  {"gpu": {"krylov": "fcg"}}, {"gpu": {"coarse-solve": "inverse"}}):
        conf = {"grid": {"periodic": [True, False, False]}}
        conf.update(extra)
        with pytest.raises(_lib.CdrError) as e:
            Solver2D(so, Config(conf))
        assert "periodic" in str(e.value)
