"""Parity of the 3D CUDA kernels and solver with the CPU oracle, through the C ABI.

Bit-exact: residual, 8-colour Gauss-Seidel (both directions), restriction,
interpolate-add, operator-induced interpolation, Galerkin coarse operator,
coarsest banded Cholesky and the whole FP64 solve (iterates identical, history
within 1e-12: only the norm's summation order differs).  FP32-refined solves
must reach the tolerance.  The same for seven-point fine operators (4 planes,
red-black Gauss-Seidel, the seven-point interpolation branch), plus the
reference's 200^3 seven-point Poisson known-answer test.
"""
import ctypes

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import gallery as G
from cedar_b200.config import Config
from tests.gpu_util import host, padded, ptr, stream

pytestmark = pytest.mark.gpu

SIZES = [(9, 9, 9), (10, 8, 7), (16, 15, 17), (33, 32, 31)]


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    return _lib.load()


def make_op3(nx, ny, nz, seed=0, sigma=1.0):
    rng = np.random.default_rng(seed + 100 * nx + 10 * ny + nz)
    return G.fe3_hetero(np.exp(sigma * rng.standard_normal((nz + 1, ny + 1, nx + 1))))


def grid3(nx, ny, nz, seed):
    rng = np.random.default_rng(seed + 7 * nx + 3 * ny + nz)
    a = np.zeros((nz + 2, ny + 2, nx + 2))
    a[1:-1, 1:-1, 1:-1] = rng.standard_normal((nz, ny, nx))
    return a


def coarse(n):
    return (n - 1) // 2 + 1


def pitch_of(nx, extra=3):
    return nx + 2 + extra


def unpad(t, nx):
    return host(t)[..., :nx + 2]


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_residual3_bitwise(lib, oracle, nx, ny, nz):
    so, x, b = make_op3(nx, ny, nz), grid3(nx, ny, nz, 1), grid3(nx, ny, nz, 2)
    p = pitch_of(nx)
    dso, dx, db, dr = padded(so, p), padded(x, p), padded(b, p), padded(np.zeros_like(x), p)
    nrm = padded(np.zeros((1, 1)), 1)
    scratch = padded(np.zeros((1, lib.cdr_gpu_norm_scratch_bytes() // 8)), lib.cdr_gpu_norm_scratch_bytes() // 8)
    _lib.check(lib.cdr_gpu_residual_3d_f64(ptr(dso), 14, ptr(dx), ptr(db), ptr(dr), nx, ny, nz, p, ptr(nrm),
                                           ptr(scratch), stream()))
    r_ref = oracle.residual3(so, x, b)
    r = unpad(dr, nx)
    assert np.array_equal(r[1:-1, 1:-1, 1:-1], r_ref[1:-1, 1:-1, 1:-1])
    assert abs(host(nrm)[0, 0] - oracle.l2norm3(r_ref)) <= 1e-13 * oracle.l2norm3(r_ref)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_gs3_bitwise(lib, oracle, nx, ny, nz):
    so, x, b = make_op3(nx, ny, nz), grid3(nx, ny, nz, 3), grid3(nx, ny, nz, 4)
    sor = oracle.setup_recip3(so)
    p = pitch_of(nx, 5)
    dso, dx, db, dsor = padded(so, p), padded(x, p), padded(b, p), padded(np.zeros_like(x), p)
    _lib.check(lib.cdr_gpu_setup_recip_3d_f64(ptr(dso), ptr(dsor), nx, ny, nz, p, stream()))
    assert np.array_equal(unpad(dsor, nx)[1:-1, 1:-1, 1:-1], sor[1:-1, 1:-1, 1:-1])
    xr = x.copy()
    for updown in (_lib.DOWN, _lib.UP, _lib.DOWN):
        oracle.relax_gs3(so, xr, b, sor, updown)
        _lib.check(lib.cdr_gpu_relax_point_3d_f64(ptr(dso), 14, ptr(dx), ptr(db), ptr(dsor), nx, ny, nz, p, updown,
                                                  stream()))
    assert np.array_equal(unpad(dx, nx), xr)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_setup_interp_galerkin3_bitwise(lib, oracle, nx, ny, nz):
    so = make_op3(nx, ny, nz, seed=5, sigma=1.5)
    nxc, nyc, nzc = coarse(nx), coarse(ny), coarse(nz)
    ci_ref = oracle.setup_interp3(so, nxc, nyc, nzc)
    soc_ref = oracle.galerkin3(so, ci_ref)
    pf, pc = pitch_of(nx), pitch_of(nxc, 6)
    dso = padded(so, pf)
    dci = padded(np.zeros((26, nzc + 2, nyc + 2, nxc + 2)), pc)
    dsoc = padded(np.zeros((14, nzc + 2, nyc + 2, nxc + 2)), pc)
    _lib.check(lib.cdr_gpu_setup_interp_3d_f64(ptr(dso), 14, ptr(dci), nx, ny, nz, pf, nxc, nyc, nzc, pc, stream()))
    _lib.check(lib.cdr_gpu_galerkin_3d_f64(ptr(dso), 14, ptr(dci), ptr(dsoc), nx, ny, nz, pf, nxc, nyc, nzc, pc,
                                           stream()))
    ci = unpad(dci, nxc)
    soc = unpad(dsoc, nxc)
    bad = [l for l in range(26) if not np.array_equal(ci[l], ci_ref[l])]
    assert not bad, "interpolation planes differ: %s" % bad
    bad = [q for q in range(14) if not np.array_equal(soc[q], soc_ref[q])]
    assert not bad, "Galerkin planes differ: %s" % bad


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_transfers3_bitwise(lib, oracle, nx, ny, nz):
    so = make_op3(nx, ny, nz, seed=6)
    nxc, nyc, nzc = coarse(nx), coarse(ny), coarse(nz)
    ci = oracle.setup_interp3(so, nxc, nyc, nzc)
    r, x = grid3(nx, ny, nz, 7), grid3(nx, ny, nz, 8)
    xc = grid3(nxc, nyc, nzc, 9)
    pf, pc = pitch_of(nx, 1), pitch_of(nxc, 2)
    dci, dr, dso, dx = padded(ci, pc), padded(r, pf), padded(so, pf), padded(x, pf)
    dbc, dxc = padded(np.zeros_like(xc), pc), padded(xc, pc)
    _lib.check(lib.cdr_gpu_restrict_3d_f64(ptr(dci), ptr(dr), ptr(dbc), nx, ny, nz, pf, nxc, nyc, nzc, pc, stream()))
    bc_ref = oracle.restrict3(ci, r)
    assert np.array_equal(unpad(dbc, nxc)[1:-1, 1:-1, 1:-1], bc_ref[1:-1, 1:-1, 1:-1])
    _lib.check(lib.cdr_gpu_interp_add_3d_f64(ptr(dci), ptr(dxc), ptr(dr), ptr(dso), ptr(dx), nx, ny, nz, pf, nxc,
                                             nyc, nzc, pc, stream()))
    x_ref = oracle.interp_add3(ci, xc, r.copy(), so, x.copy())
    assert np.array_equal(unpad(dx, nx), x_ref)
    assert np.array_equal(unpad(dr, nx), r)  # the residual argument is not modified


@pytest.mark.parametrize("n", [(3, 3, 3), (4, 3, 5), (7, 6, 5)])
def test_coarse_cholesky3_bitwise(lib, oracle, n):
    nx, ny, nz = n
    so = make_op3(nx, ny, nz, seed=9)
    b = grid3(nx, ny, nz, 10)
    abd_ref, info = oracle.setup_cg3(so)
    assert info == 0
    x_ref = oracle.solve_cg3(abd_ref, b)
    import torch
    p = pitch_of(nx, 4)
    dso, db, dx = padded(so, p), padded(b, p), padded(np.zeros_like(b), p)
    ldab = nx * (ny + 1) + 2
    dabd = torch.zeros(ldab * nx * ny * nz, dtype=torch.float64, device="cuda")
    dinfo = torch.ones(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.cdr_gpu_setup_cg_3d_f64(ptr(dso), 14, nx, ny, nz, p, ptr(dabd), ptr(dinfo), stream()))
    _lib.check(lib.cdr_gpu_solve_cg_3d_f64(ptr(dabd), ptr(dx), ptr(db), nx, ny, nz, p, stream()))
    assert int(dinfo.cpu()[0]) == 0
    assert np.array_equal(host(dabd).reshape(abd_ref.shape), abd_ref)
    assert np.array_equal(unpad(dx, nx)[1:-1, 1:-1, 1:-1], x_ref[1:-1, 1:-1, 1:-1])


def _rhs3(nx, ny, nz, seed=12):
    rng = np.random.default_rng(seed)
    b = np.zeros((nz + 2, ny + 2, nx + 2))
    b[1:-1, 1:-1, 1:-1] = rng.uniform(0, 1, (nz, ny, nx)) / (nx + 1) ** 3
    return b


@pytest.mark.parametrize("nx,ny,nz,graph", [(15, 15, 15, True), (16, 15, 17, True), (31, 33, 30, False),
                                            (63, 63, 63, True)])
def test_solver3_matches_oracle(lib, oracle, nx, ny, nz, graph):
    from cedar_b200.solver import Solver3D
    so = make_op3(nx, ny, nz, seed=11, sigma=1.5)
    b = _rhs3(nx, ny, nz)
    conf = Config({"solver": {"max-iter": 25, "tol": 1e-10}, "gpu": {"graph": graph}})
    s = Solver3D(so, conf)
    ref = oracle.Solver3(so, maxiter=25, tol=1e-10)
    assert s.nlevels == ref.nlevels
    for l in range(1, s.nlevels):
        assert np.array_equal(s.level_array(l, "so"), ref.level_array(l, "so")), "level %d operator" % l
        assert np.array_equal(s.level_array(l, "ci"), ref.level_array(l, "ci")), "level %d interpolation" % l
    x = s.solve(b)
    x_ref, h_ref = ref.solve(b)
    assert len(s.history) == len(h_ref)
    assert np.abs(s.history - h_ref).max() <= 1e-12 * max(1.0, h_ref.max())
    assert np.array_equal(x, x_ref)
    assert h_ref[-1] < 1e-10


@pytest.mark.parametrize("nx,ny,nz", [(31, 31, 31), (40, 33, 35)])
def test_solver3_fp32_ir_reaches_tol(lib, oracle, nx, ny, nz):
    from cedar_b200.solver import Solver3D
    so = make_op3(nx, ny, nz, seed=13, sigma=2.0)
    b = _rhs3(nx, ny, nz, seed=14)
    s = Solver3D(so, Config({"solver": {"max-iter": 30, "tol": 1e-10}, "gpu": {"precision": "fp32-ir"}}))
    x = s.solve(b)
    assert s.history[-1] < 1e-10
    r = oracle.residual3(so, x, b)
    assert oracle.l2norm3(r) / oracle.l2norm3(b) < 1e-10
    ref = oracle.Solver3(so, maxiter=30, tol=1e-10)
    _, h_ref = ref.solve(b)
    assert len(s.history) <= len(h_ref) + 2


@pytest.mark.parametrize("nx,ny,nz,relax", [(15, 15, 15, "point"), (31, 33, 30, "point"), (15, 13, 16, "plane-xyz")])
def test_solver3_fcycle_matches_oracle(lib, oracle, nx, ny, nz, relax):
    """solver.cycle.type = f on the 3D solver (cycle::fcycle): every cycle
    restarts from the restricted right-hand sides, as in the reference; FP64
    iterate and history bit-identical to the oracle's F-cycle (sequential line
    substitutions inside the plane solves)."""
    from cedar_b200.solver import Solver3D
    so = make_op3(nx, ny, nz, seed=17, sigma=1.5)
    b = _rhs3(nx, ny, nz, seed=18)
    gpu = {"line-solve": "sequential"} if relax != "point" else {}
    s = Solver3D(so, Config({"solver": {"relaxation": relax, "max-iter": 3, "tol": 1e-30, "cycle": {"type": "f"}},
                             "gpu": gpu}))
    x = s.solve(b)
    x_ref, h_ref = oracle.Solver3(so, maxiter=3, tol=1e-30, relax=relax, cycle="f").solve(b)
    assert np.array_equal(x, x_ref)
    assert np.abs(s.history - h_ref).max() <= 1e-12 * max(1.0, h_ref.max())
    assert h_ref[0] < 0.5 and np.all(h_ref == h_ref[0])  # the F-cycle ignores the incoming x


def test_solver3_rejects_unsupported(lib):
    from cedar_b200.solver import Solver3D
    so = make_op3(7, 7, 7)
    with pytest.raises(NotImplementedError):
        Solver3D(so, Config({"solver": {"relaxation": "line-x"}}))
    s = _lib.Settings()
    lib.cdr_gpu_settings_default(ctypes.byref(s))
    s.relaxation = 1
    h = ctypes.c_void_p()
    rc = lib.cdr_gpu_solver3_create(ctypes.byref(s), so.ctypes.data, 14, 7, 7, 7, None, ctypes.byref(h))
    assert rc == 7  # CDR_ERR_UNSUPPORTED


@pytest.mark.parametrize("n", [(7, 7, 7), (12, 9, 10), (31, 31, 31)])
def test_fe_assemble3_bitwise_and_device_create(lib, oracle, n):
    import torch
    from cedar_b200.solver import Solver3D
    nx, ny, nz = n
    rng = np.random.default_rng(nx * ny * nz)
    k = np.exp(1.5 * rng.standard_normal((nz + 1, ny + 1, nx + 1)))
    so_ref = G.fe3_hetero(k)
    p = pitch_of(nx, 7)
    dk = torch.from_numpy(k).cuda()
    dso = torch.full((14, nz + 2, ny + 2, p), 7.0, dtype=torch.float64, device="cuda")
    _lib.check(lib.cdr_gpu_fe_assemble_3d_f64(ptr(dk), nx + 1, (nx + 1) * (ny + 1), ptr(dso), nx, ny, nz, p,
                                              stream()))
    assert np.array_equal(unpad(dso, nx), so_ref)
    if nx == ny == nz:
        b = _rhs3(nx, ny, nz, seed=15)
        conf = Config({"solver": {"max-iter": 30, "tol": 1e-10}})
        s = Solver3D(dso.data_ptr(), conf, stream=0, dims=(nx, ny, nz), pitch=p)
        x = s.solve(b)
        x_ref, h_ref = oracle.Solver3(so_ref, maxiter=30, tol=1e-10).solve(b)
        assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("nx,ny,nz", [(15, 15, 15), (16, 13, 11), (23, 20, 26)])
def test_solver3_plane_relaxation_matches_oracle(lib, oracle, nx, ny, nz):
    """Plane relaxation (one batched 2D line-xy V-cycle per plane, red-black over
    planes, xy/yz/xz going down): with the sequential line substitutions every
    operation follows the oracle, so the iterates are identical."""
    from cedar_b200.solver import Solver3D
    so = make_op3(nx, ny, nz, seed=16, sigma=1.5)
    b = _rhs3(nx, ny, nz, seed=17)
    conf = Config({"solver": {"relaxation": "plane-xyz", "max-iter": 12, "tol": 1e-10},
                   "gpu": {"line-solve": "sequential"}})
    s = Solver3D(so, conf)
    ref = oracle.Solver3(so, maxiter=12, tol=1e-10, relax="plane-xyz")
    x = s.solve(b)
    x_ref, h_ref = ref.solve(b)
    assert len(s.history) == len(h_ref)
    assert np.abs(s.history - h_ref).max() <= 1e-12 * max(1.0, h_ref.max())
    assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("relax", ["plane-xy", "plane-xz", "plane-yz"])
def test_solver3_single_plane_direction_matches_oracle(lib, oracle, relax):
    from cedar_b200.solver import Solver3D
    nx, ny, nz = 14, 17, 12
    so = make_op3(nx, ny, nz, seed=18)
    b = _rhs3(nx, ny, nz, seed=19)
    conf = Config({"solver": {"relaxation": relax, "max-iter": 4, "tol": 1e-12},
                   "gpu": {"line-solve": "sequential", "graph": False}})
    x = Solver3D(so, conf).solve(b)
    x_ref, _ = oracle.Solver3(so, maxiter=4, tol=1e-12, relax=relax).solve(b)
    assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("prec", ["fp64", "fp32-ir"])
def test_solver3_plane_relaxation_fast_path_reaches_tol(lib, oracle, prec):
    """Default (parallel-scan) line substitutions and the FP32 cycle: same
    convergence as the oracle to within a cycle or two."""
    from cedar_b200.solver import Solver3D
    n = 31
    so = make_op3(n, n, n, seed=20, sigma=1.5)
    b = _rhs3(n, n, n, seed=21)
    s = Solver3D(so, Config({"solver": {"relaxation": "plane-xyz", "max-iter": 20, "tol": 1e-10},
                             "gpu": {"precision": prec}}))
    x = s.solve(b)
    _, h_ref = oracle.Solver3(so, maxiter=20, tol=1e-10, relax="plane-xyz").solve(b)
    assert s.history[-1] < 1e-10
    assert len(s.history) <= len(h_ref) + 2
    r = oracle.residual3(so, x, b)
    assert oracle.l2norm3(r) / oracle.l2norm3(b) < 1e-10


# ------------------------------------------------------- seven-point operators
def make_op7(nx, ny, nz, seed=0, sigma=1.0):
    rng = np.random.default_rng(seed + 100 * nx + 10 * ny + nz)
    return G.fd3_hetero(np.exp(sigma * rng.standard_normal((nz + 2, ny + 2, nx + 2))))


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_seven_point_residual_gs_bitwise(lib, oracle, nx, ny, nz):
    so, x, b = make_op7(nx, ny, nz), grid3(nx, ny, nz, 21), grid3(nx, ny, nz, 22)
    p = pitch_of(nx, 2)
    dso, dx, db, dr = padded(so, p), padded(x, p), padded(b, p), padded(np.zeros_like(x), p)
    nrm = padded(np.zeros((1, 1)), 1)
    scratch = padded(np.zeros((1, lib.cdr_gpu_norm_scratch_bytes() // 8)), lib.cdr_gpu_norm_scratch_bytes() // 8)
    _lib.check(lib.cdr_gpu_residual_3d_f64(ptr(dso), 4, ptr(dx), ptr(db), ptr(dr), nx, ny, nz, p, ptr(nrm),
                                           ptr(scratch), stream()))
    r_ref = oracle.residual3(so, x, b)
    assert np.array_equal(unpad(dr, nx)[1:-1, 1:-1, 1:-1], r_ref[1:-1, 1:-1, 1:-1])
    assert abs(host(nrm)[0, 0] - oracle.l2norm3(r_ref)) <= 1e-13 * oracle.l2norm3(r_ref)
    sor = oracle.setup_recip3(so)
    dsor = padded(np.zeros_like(x), p)
    _lib.check(lib.cdr_gpu_setup_recip_3d_f64(ptr(dso), ptr(dsor), nx, ny, nz, p, stream()))
    xr = x.copy()
    for updown in (_lib.DOWN, _lib.UP, _lib.UP, _lib.DOWN):
        oracle.relax_gs3(so, xr, b, sor, updown)
        _lib.check(lib.cdr_gpu_relax_point_3d_f64(ptr(dso), 4, ptr(dx), ptr(db), ptr(dsor), nx, ny, nz, p, updown,
                                                  stream()))
    assert np.array_equal(unpad(dx, nx), xr)


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_seven_point_interp_galerkin_bitwise(lib, oracle, nx, ny, nz):
    so = make_op7(nx, ny, nz, seed=23, sigma=1.5)
    nxc, nyc, nzc = coarse(nx), coarse(ny), coarse(nz)
    ci_ref = oracle.setup_interp3(so, nxc, nyc, nzc)
    soc_ref = oracle.galerkin3(so, ci_ref)
    pf, pc = pitch_of(nx, 4), pitch_of(nxc, 1)
    dso = padded(so, pf)
    dci = padded(np.zeros((26, nzc + 2, nyc + 2, nxc + 2)), pc)
    dsoc = padded(np.zeros((14, nzc + 2, nyc + 2, nxc + 2)), pc)
    _lib.check(lib.cdr_gpu_setup_interp_3d_f64(ptr(dso), 4, ptr(dci), nx, ny, nz, pf, nxc, nyc, nzc, pc, stream()))
    _lib.check(lib.cdr_gpu_galerkin_3d_f64(ptr(dso), 4, ptr(dci), ptr(dsoc), nx, ny, nz, pf, nxc, nyc, nzc, pc,
                                           stream()))
    ci, soc = unpad(dci, nxc), unpad(dsoc, nxc)
    bad = [l for l in range(26) if not np.array_equal(ci[l], ci_ref[l])]
    assert not bad, "interpolation planes differ: %s" % bad
    bad = [q for q in range(14) if not np.array_equal(soc[q], soc_ref[q])]
    assert not bad, "Galerkin planes differ: %s" % bad


def test_seven_point_coarse_cholesky_bitwise(lib, oracle):
    import torch
    nx, ny, nz = 5, 4, 6
    so = make_op7(nx, ny, nz, seed=24)
    b = grid3(nx, ny, nz, 25)
    abd_ref, info = oracle.setup_cg3(so)
    assert info == 0
    x_ref = oracle.solve_cg3(abd_ref, b)
    p = pitch_of(nx, 3)
    dso, db, dx = padded(so, p), padded(b, p), padded(np.zeros_like(b), p)
    dabd = torch.zeros((nx * (ny + 1) + 2) * nx * ny * nz, dtype=torch.float64, device="cuda")
    dinfo = torch.ones(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.cdr_gpu_setup_cg_3d_f64(ptr(dso), 4, nx, ny, nz, p, ptr(dabd), ptr(dinfo), stream()))
    _lib.check(lib.cdr_gpu_solve_cg_3d_f64(ptr(dabd), ptr(dx), ptr(db), nx, ny, nz, p, stream()))
    assert int(dinfo.cpu()[0]) == 0
    assert np.array_equal(host(dabd).reshape(abd_ref.shape), abd_ref)
    assert np.array_equal(unpad(dx, nx)[1:-1, 1:-1, 1:-1], x_ref[1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("relax,n", [("point", (15, 15, 15)), ("point", (31, 30, 33)), ("plane-xyz", (15, 15, 15)),
                                     ("plane-xyz", (16, 13, 19))])
def test_seven_point_solver3_matches_oracle(lib, oracle, relax, n):
    from cedar_b200.solver import Solver3D
    nx, ny, nz = n
    so = make_op7(nx, ny, nz, seed=26, sigma=1.5)
    b = _rhs3(nx, ny, nz, seed=27)
    conf = Config({"solver": {"relaxation": relax, "max-iter": 40, "tol": 1e-10}, "gpu": {"line-solve": "sequential"}})
    s = Solver3D(so, conf)
    ref = oracle.Solver3(so, maxiter=40, tol=1e-10, relax=relax)
    assert s.nlevels == ref.nlevels
    assert np.array_equal(s.level_array(0, "so"), so)
    for l in range(1, s.nlevels):
        assert np.array_equal(s.level_array(l, "so"), ref.level_array(l, "so")), "level %d operator" % l
    x = s.solve(b)
    x_ref, h_ref = ref.solve(b)
    assert len(s.history) == len(h_ref)
    assert np.abs(s.history - h_ref).max() <= 1e-12 * max(1.0, h_ref.max())
    assert np.array_equal(x, x_ref)
    assert h_ref[-1] < 1e-10


@pytest.mark.parametrize("relax", ["point", "plane-xyz"])
def test_seven_point_solver3_fp32_ir_reaches_tol(lib, oracle, relax):
    from cedar_b200.solver import Solver3D
    n = 31
    so = make_op7(n, n, n, seed=28, sigma=1.0)  # sigma 2: 57 FP64 point cycles to 1e-10
    b = _rhs3(n, n, n, seed=29)
    s = Solver3D(so, Config({"solver": {"relaxation": relax, "max-iter": 30, "tol": 1e-10},
                             "gpu": {"precision": "fp32-ir"}}))
    x = s.solve(b)
    assert s.history[-1] < 1e-10
    r = oracle.residual3(so, x, b)
    assert oracle.l2norm3(r) / oracle.l2norm3(b) < 1e-10
    _, h_ref = oracle.Solver3(so, maxiter=30, tol=1e-10, relax=relax).solve(b)
    assert len(s.history) <= len(h_ref) + 2


def test_seven_point_poisson_known_answer_200(lib, oracle):
    """test/3d/test_poisson.cc:73-104 (SerialPoisson3.Isotropic) at its own size:
    200^3 seven-point Poisson, default settings; ||r||_2 < 1e-8 and the error
    against sin(2 pi x) sin(2 pi y) sin(2 pi z) below 1e-4."""
    from cedar_b200.solver import Solver3D
    n = 200
    so = G.poisson3(n, n, n)
    b = G.poisson3_rhs_sin2pi(n, n, n)
    s = Solver3D(so, Config({}))
    x = s.solve(b)
    r = oracle.residual3(so, x, b)
    assert oracle.l2norm3(r) < 1e-8
    assert np.abs(x - G.poisson3_exact_sin2pi(n, n, n))[1:-1, 1:-1, 1:-1].max() < 1e-4


def test_solver3_rejects_bad_nstencil(lib):
    so = make_op7(7, 7, 7)
    s = _lib.Settings()
    lib.cdr_gpu_settings_default(ctypes.byref(s))
    h = ctypes.c_void_p()
    assert lib.cdr_gpu_solver3_create(ctypes.byref(s), so.ctypes.data, 5, 7, 7, 7, None, ctypes.byref(h)) == 1
