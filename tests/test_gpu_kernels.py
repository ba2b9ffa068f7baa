"""Parity of every 2D CUDA kernel with the CPU oracle, through the C ABI.

Bit-exact: residual, point Gauss-Seidel, restriction, interpolate-add,
interpolation setup, Galerkin coarse operator, line factorization, line
relaxation with sequential substitutions, and the coarsest Cholesky (same
operand order, no FMA).  Tolerances: line relaxation with the parallel-scan
substitutions 1e-12, FP32 kernels 1e-5 relative to the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import gallery as G
from cedar_b200 import problems as P
from tests.gpu_util import dev, host, padded, ptr, rel_err, stream

pytestmark = pytest.mark.gpu

SIZES = [(9, 9, 3), (10, 8, 3), (17, 12, 5), (32, 33, 5), (63, 64, 5), (64, 63, 3), (130, 97, 5)]


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    return _lib.load()


def make_op(nx, ny, ns, seed=0):
    rng = np.random.default_rng(seed + 7 * nx + ny)
    if ns == 3:
        so = G.diag_diffusion(nx, ny, 1.0, 0.5)
        so[1:] *= 1 + 0.5 * rng.random(so[1:].shape)
        so[1, :, :2] = 0; so[2, :2, :] = 0; so[:, 0, :] = 0; so[:, :, 0] = 0
        so[:, -1, :] = 0; so[:, :, -1] = 0
        so[0, 1:-1, 1:-1] = 2.2 * (so[1, 1:-1, 1:-1] + so[1, 1:-1, 2:] + so[2, 1:-1, 1:-1] + so[2, 2:, 1:-1]) / 2
        so[0, 1:-1, 1:-1] += 0.1
    else:
        kx, ky = P.hetero_coefficients(nx if nx == ny else max(nx, ny), sigma=1.0, n_incl=3, contrast=50.0,
                                       aniso=0.3, seed_field=seed + 11, seed_incl=seed + 12)
        so = G.fe_hetero(kx[:ny + 1, :nx + 1], ky[:ny + 1, :nx + 1])
    return np.ascontiguousarray(so)


def grid(nx, ny, seed=1):
    rng = np.random.default_rng(seed + nx * 3 + ny)
    a = np.zeros((ny + 2, nx + 2))
    a[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    return a


@pytest.mark.parametrize("nx,ny,ns", SIZES)
def test_residual_bitwise_and_norm(lib, oracle, nx, ny, ns):
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 1), grid(nx, ny, 2)
    r_ref = oracle.residual(so, x, b)
    dso, dx, db = dev(so), dev(x), dev(b)
    dr = dev(np.zeros_like(x))
    nrm = dev(np.zeros(1))
    scratch = dev(np.zeros(lib.cdr_gpu_norm_scratch_bytes() // 8))
    _lib.check(lib.cdr_gpu_residual_2d_f64(ptr(dso), ns, ptr(dx), ptr(db), ptr(dr), nx, ny, nx + 2, ptr(nrm),
                                           ptr(scratch), stream()))
    np.testing.assert_array_equal(host(dr), r_ref)
    assert abs(host(nrm)[0] - oracle.l2norm(r_ref)) <= 1e-13 * oracle.l2norm(r_ref)


@pytest.mark.parametrize("nx,ny,ns", SIZES[:4])
def test_residual_padded_pitch_and_f32(lib, oracle, nx, ny, ns):
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 1), grid(nx, ny, 2)
    r_ref = oracle.residual(so, x, b)
    pitch = ((nx + 2 + 31) // 32) * 32
    dso, dx, db = padded(so, pitch), padded(x, pitch), padded(b, pitch)
    dr = padded(np.zeros_like(x), pitch)
    _lib.check(lib.cdr_gpu_residual_2d_f64(ptr(dso), ns, ptr(dx), ptr(db), ptr(dr), nx, ny, pitch, None, None,
                                           stream()))
    np.testing.assert_array_equal(host(dr)[:, :nx + 2], r_ref)
    import torch
    fso, fx, fb = dso.float(), dx.float(), db.float()  # held: pointers below stay valid
    fr = torch.zeros_like(fx)
    _lib.check(lib.cdr_gpu_residual_2d_f32(ptr(fso), ns, ptr(fx), ptr(fb), ptr(fr), nx, ny, pitch, None, None,
                                           stream()))
    assert rel_err(host(fr)[:, :nx + 2], r_ref) < 1e-5


@pytest.mark.parametrize("nx,ny,ns", SIZES)
@pytest.mark.parametrize("updown", [0, 1])
def test_point_relax_bitwise(lib, oracle, nx, ny, ns, updown):
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 3), grid(nx, ny, 4)
    sor = oracle.setup_recip(so)
    xr = x.copy()
    for _ in range(2):
        oracle.relax_gs(so, xr, b, sor, updown)
    dso, dx, db = dev(so), dev(x), dev(b)
    dsor = dev(np.zeros_like(x))
    _lib.check(lib.cdr_gpu_setup_recip_2d_f64(ptr(dso), ptr(dsor), nx, ny, nx + 2, stream()))
    np.testing.assert_array_equal(host(dsor), sor[1])
    for _ in range(2):
        _lib.check(lib.cdr_gpu_relax_point_2d_f64(ptr(dso), ns, ptr(dx), ptr(db), ptr(dsor), nx, ny, nx + 2, updown,
                                                  stream()))
    np.testing.assert_array_equal(host(dx), xr)


@pytest.mark.parametrize("nx,ny,ns", SIZES)
def test_interp_setup_transfer_and_galerkin(lib, oracle, nx, ny, ns):
    so = make_op(nx, ny, ns)
    nxc, nyc = (nx - 1) // 2 + 1, (ny - 1) // 2 + 1
    ci = oracle.setup_interp(so, nxc, nyc)
    soc = oracle.galerkin(so, ci)
    dso = dev(so)
    dci = dev(np.zeros_like(ci))
    _lib.check(lib.cdr_gpu_setup_interp_2d_f64(ptr(dso), ns, ptr(dci), nx, ny, nx + 2, nxc, nyc, nxc + 2, stream()))
    np.testing.assert_array_equal(host(dci), ci)
    dsoc = dev(np.zeros_like(soc))
    _lib.check(lib.cdr_gpu_galerkin_2d_f64(ptr(dso), ns, ptr(dci), ptr(dsoc), nx, ny, nx + 2, nxc, nyc, nxc + 2,
                                           stream()))
    np.testing.assert_array_equal(host(dsoc), soc)
    # restriction and interpolate-add
    r = grid(nx, ny, 5)
    bc = oracle.restrict(ci, r)
    dbc = dev(np.zeros_like(bc))
    dr = dev(r)
    _lib.check(lib.cdr_gpu_restrict_2d_f64(ptr(dci), ptr(dr), ptr(dbc), nx, ny, nx + 2, nxc, nyc, nxc + 2,
                                           stream()))
    np.testing.assert_array_equal(host(dbc), bc)
    xc = grid(nxc, nyc, 6)
    x = grid(nx, ny, 7)
    xr = x.copy()
    oracle.interp_add(ci, xc, r.copy(), so, xr)
    dx, dxc = dev(x), dev(xc)
    _lib.check(lib.cdr_gpu_interp_add_2d_f64(ptr(dci), ptr(dxc), ptr(dr), ptr(dso), ptr(dx), nx, ny,
                                             nx + 2, nxc, nyc, nxc + 2, stream()))
    np.testing.assert_array_equal(host(dx), xr)
    # FP32 transfer kernels
    import torch
    fbc = torch.zeros_like(dbc).float()
    fci, fr = dci.float(), dr.float()
    _lib.check(lib.cdr_gpu_restrict_2d_f32(ptr(fci), ptr(fr), ptr(fbc), nx, ny, nx + 2, nxc, nyc,
                                           nxc + 2, stream()))
    assert rel_err(host(fbc), bc) < 1e-5


@pytest.mark.parametrize("nx,ny,ns", SIZES)
@pytest.mark.parametrize("updown", [0, 1])
def test_line_relax(lib, oracle, nx, ny, ns, updown):
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 8), grid(nx, ny, 9)
    sx, ix = oracle.setup_lines_x(so)
    sy, iy = oracle.setup_lines_y(so)
    assert ix == 0 and iy == 0
    dso = dev(so)
    info = dev(np.zeros(2, dtype=np.int32))
    dsx = dev(np.zeros_like(sx))
    dsy = dev(np.zeros_like(sy))
    _lib.check(lib.cdr_gpu_setup_lines_2d_f64(ptr(dso), ns, ptr(dsx), nx, ny, nx + 2, ny + 2, _lib.DIR_X, ptr(info),
                                              stream()))
    _lib.check(lib.cdr_gpu_setup_lines_2d_f64(ptr(dso), ns, ptr(dsy), nx, ny, nx + 2, ny + 2, _lib.DIR_Y, ptr(info),
                                              stream()))
    np.testing.assert_array_equal(host(dsx)[:, 1:-1, 1:-1], sx[:, 1:-1, 1:-1])
    np.testing.assert_array_equal(host(dsy)[:, 1:-1, 1:-1], sy[:, 1:-1, 1:-1])
    assert (host(info) == 0).all()
    for direction, sor, dsor, fn in ((_lib.DIR_X, sx, dsx, oracle.relax_lines_x), (_lib.DIR_Y, sy, dsy, oracle.relax_lines_y)):
        xr = x.copy()
        fn(so, xr, b, sor, updown)
        fn(so, xr, b, sor, 1 - updown)
        dx, dbb = dev(x), dev(b)
        for ud in (updown, 1 - updown):
            _lib.check(lib.cdr_gpu_relax_lines_2d_f64(ptr(dso), ns, ptr(dx), ptr(dbb), ptr(dsor), nx, ny, nx + 2,
                                                      ny + 2, direction, ud, 0, stream()))
        assert rel_err(host(dx), xr) < 1e-12, direction
        dxe = dev(x)
        for ud in (updown, 1 - updown):
            _lib.check(lib.cdr_gpu_relax_lines_2d_f64(ptr(dso), ns, ptr(dxe), ptr(dbb), ptr(dsor), nx, ny, nx + 2,
                                                      ny + 2, direction, ud, _lib.LINES_EXACT, stream()))
        np.testing.assert_array_equal(host(dxe), xr)
        # FP32 factors and sweep
        fs = dev(np.zeros_like(sor)).float()
        _lib.check(lib.cdr_gpu_setup_lines_2d_f32(ptr(dso), ns, ptr(fs), nx, ny, nx + 2, ny + 2, direction, ptr(info),
                                                  stream()))
        fx, fso, fb = dev(x).float(), dso.float(), dbb.float()
        for ud in (updown, 1 - updown):
            _lib.check(lib.cdr_gpu_relax_lines_2d_f32(ptr(fso), ns, ptr(fx), ptr(fb), ptr(fs), nx,
                                                      ny, nx + 2, ny + 2, direction, ud, 0, stream()))
        assert rel_err(host(fx), xr) < 1e-4, direction


LINE_SIZES = [(9, 9, 3), (17, 12, 5), (64, 63, 3), (130, 97, 5), (255, 31, 5), (31, 255, 5), (1023, 20, 5),
              (20, 1023, 5), (2047, 12, 5), (12, 2047, 5), (2047, 9, 3), (9, 2047, 3),
              # line lengths n = 2^k: the last thread of a line owns the tail point
              (8, 16, 5), (128, 33, 5), (33, 256, 5), (1024, 9, 5), (9, 1024, 5), (512, 512, 3)]


@pytest.mark.parametrize("nx,ny,ns", LINE_SIZES)
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_line_relax_register_chunk_kernel(lib, oracle, nx, ny, ns, precision):
    """Padded pitches (multiples of 32) select the register-chunk sweep kernel."""
    import torch
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 8), grid(nx, ny, 9)
    sx, _ = oracle.setup_lines_x(so)
    sy, _ = oracle.setup_lines_y(so)
    pitch = ((nx + 2 + 31) // 32) * 32
    tpitch = ((ny + 2 + 31) // 32) * 32
    dt = torch.float64 if precision == "f64" else torch.float32
    fn = lib.cdr_gpu_relax_lines_2d_f64 if precision == "f64" else lib.cdr_gpu_relax_lines_2d_f32
    dso = padded(so, pitch, dt)
    dbb = padded(b, pitch, dt)
    gx, gy = sx, sy
    if precision == "f32":  # FP32 factors hold reciprocal pivots
        gx, gy = sx.copy(), sy.copy()
        gx[0][1:-1, 1:-1] = 1.0 / sx[0][1:-1, 1:-1]
        gy[0][1:-1, 1:-1] = 1.0 / sy[0][1:-1, 1:-1]
    dsx = padded(gx, pitch, dt)
    dsy = padded(gy, tpitch, dt)
    for direction, sor, dsor, ofn in ((_lib.DIR_X, sx, dsx, oracle.relax_lines_x), (_lib.DIR_Y, sy, dsy, oracle.relax_lines_y)):
        for updown in (0, 1):
            xr = x.copy()
            ofn(so, xr, b, sor, updown)
            dx = padded(x, pitch, dt)
            _lib.check(fn(ptr(dso), ns, ptr(dx), ptr(dbb), ptr(dsor), nx, ny, pitch, tpitch, direction, updown, 0,
                          stream()))
            got = host(dx)[:, :nx + 2]
            tol = 1e-12 if precision == "f64" else 2e-4
            assert rel_err(got, xr) < tol, (direction, updown, rel_err(got, xr))
            np.testing.assert_array_equal(got[0], 0.0)
            np.testing.assert_array_equal(got[-1], 0.0)
            np.testing.assert_array_equal(got[:, 0], 0.0)
            np.testing.assert_array_equal(got[:, nx + 1], 0.0)


STREAM_SIZES = [("f32", 256, 5000, 5), ("f32", 300, 3000, 3), ("f32", 1024, 1500, 5), ("f32", 2047, 700, 5),
                ("f32", 512, 37, 5), ("f64", 256, 5000, 5), ("f64", 1024, 1500, 5), ("f64", 700, 900, 3)]


@pytest.mark.parametrize("precision,nx,ny,ns", STREAM_SIZES)
def test_streamed_x_lines(lib, oracle, precision, nx, ny, ns):
    """CDR_LINES_STREAM: the persistent x-line kernel whose rows arrive in shared
    memory by bulk copies two lines ahead.  Enough lines that every CTA reuses
    both stages several times; FP32 results bit-identical to the default kernel
    (same elements per thread), both precisions at the oracle's rounding level."""
    import torch
    rng = np.random.default_rng(nx + 7 * ny)
    if ns == 3:
        so = G.diag_diffusion(nx, ny, 1.0, 0.3)
        so[1:, 1:-1, 1:-1] *= 1 + 0.5 * rng.random((2, ny, nx))
        so[1, :, :2] = 0; so[2, :2, :] = 0
        so[0, 1:-1, 1:-1] = 2.2 * (so[1, 1:-1, 1:-1] + so[1, 1:-1, 2:] + so[2, 1:-1, 1:-1] + so[2, 2:, 1:-1]) / 2 + 0.1
    else:
        so = G.fe_hetero(np.exp(rng.standard_normal((ny + 1, nx + 1))), np.exp(rng.standard_normal((ny + 1, nx + 1))))
    so = np.ascontiguousarray(so)
    x, b = grid(nx, ny, 3), grid(nx, ny, 4)
    sx, _ = oracle.setup_lines_x(so)
    pitch = ((nx + 2 + 31) // 32) * 32
    dt = torch.float64 if precision == "f64" else torch.float32
    fn = lib.cdr_gpu_relax_lines_2d_f64 if precision == "f64" else lib.cdr_gpu_relax_lines_2d_f32
    gx = sx
    if precision == "f32":
        gx = sx.copy()
        gx[0][1:-1, 1:-1] = 1.0 / sx[0][1:-1, 1:-1]
    dso, dbb, dsx = padded(so, pitch, dt), padded(b, pitch, dt), padded(gx, pitch, dt)
    for updown in (0, 1):
        xr = x.copy()
        oracle.relax_lines_x(so, xr, b, sx, updown)
        got = {}
        for flags in (_lib.LINES_STREAM, _lib.LINES_NOTUNE):
            dx = padded(x, pitch, dt)
            _lib.check(fn(ptr(dso), ns, ptr(dx), ptr(dbb), ptr(dsx), nx, ny, pitch, pitch, _lib.DIR_X, updown, flags,
                          stream()))
            got[flags] = host(dx)[:, :nx + 2]
        g = got[_lib.LINES_STREAM]
        tol = 1e-12 if precision == "f64" else 2e-4
        assert rel_err(g, xr) < tol, (updown, rel_err(g, xr))
        if precision == "f32":
            np.testing.assert_array_equal(g, got[_lib.LINES_NOTUNE])
        np.testing.assert_array_equal(g[0], 0.0)
        np.testing.assert_array_equal(g[-1], 0.0)
        np.testing.assert_array_equal(g[:, 0], 0.0)
        np.testing.assert_array_equal(g[:, nx + 1], 0.0)
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0  # no CTA gave up waiting


def test_line_setup_reports_nonpositive_pivot(lib):
    nx = ny = 8
    so = G.diag_diffusion(nx, ny, 1.0, 1.0)
    so[0, 4, 3] = -1.0  # negative diagonal on line j=4
    info = dev(np.zeros(2, dtype=np.int32))
    dsx = dev(np.zeros((2, ny + 2, nx + 2)))
    dso = dev(so)
    _lib.check(lib.cdr_gpu_setup_lines_2d_f64(ptr(dso), 3, ptr(dsx), nx, ny, nx + 2, ny + 2, _lib.DIR_X,
                                              ptr(info), stream()))
    assert host(info)[0] == 4


@pytest.mark.parametrize("n", [3, 4, 5, 7])
def test_coarse_cholesky_bitwise(lib, oracle, n):
    so = make_op(n, n, 5)
    abd, info = oracle.setup_cg(so)
    assert info == 0
    b = grid(n, n, 10)
    x = oracle.solve_cg(abd, b)
    dabd = dev(np.zeros_like(abd))
    dinfo = dev(np.zeros(1, dtype=np.int32))
    dso = dev(so)
    _lib.check(lib.cdr_gpu_setup_cg_2d_f64(ptr(dso), 5, n, n, n + 2, ptr(dabd), ptr(dinfo), stream()))
    np.testing.assert_array_equal(host(dabd), abd)
    assert host(dinfo)[0] == 0
    dx, db = dev(np.zeros_like(b)), dev(b)
    _lib.check(lib.cdr_gpu_solve_cg_2d_f64(ptr(dabd), ptr(dx), ptr(db), n, n, n + 2, stream()))
    np.testing.assert_array_equal(host(dx), x)


def test_line_autotuner_records_shapes_and_keeps_results():
    """The setup-time autotuner records a launch shape for every swept level,
    and the tuned FP32 solve is the default-shape one bit for bit: the chunks
    of a line (K per thread) are fixed by its length and the scan's tree by the
    chunk indices, so the shape changes only the timing."""
    import ctypes
    from cedar_b200 import _lib
    from cedar_b200 import problems as P
    from cedar_b200.config import Config
    from cedar_b200.solver import Solver2D
    lib = _lib.load()
    n = 255
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
    res = {}
    for tune in (True, False):
        s = Solver2D(so, Config({"solver": {"relaxation": "line-xy", "max-iter": 30, "tol": 1e-9},
                                 "gpu": {"precision": "fp32-ir", "autotune": tune}}))
        x = s.solve(b)
        res[tune] = (x, s.history.copy())
        if tune:
            for l in range(s.nlevels - 1):
                _, nx, ny, *_ = s.level_info(l, "so")
                if nx <= 32:
                    break  # fused coarse levels do not use the line kernels
                for d, (nn, nl) in ((0, (nx, ny)), (1, (ny, nx))):
                    K, cap = ctypes.c_int(), ctypes.c_int()
                    rc = lib.cdr_gpu_lines_shape(d, 1, 5, nn, nl, 0, ctypes.byref(K), ctypes.byref(cap))
                    assert rc == 0, (l, d)
                    assert K.value == 8 and cap.value in (0, 32, 64, 128, 256, 512, 1024)
    assert res[True][1][-1] < 1e-9
    np.testing.assert_array_equal(res[True][1], res[False][1])
    np.testing.assert_array_equal(res[True][0], res[False][0])


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("n", [100, 383, 1024, 2047])
def test_line_sweep_bits_independent_of_launch_shape(lib, oracle, precision, n):
    """Every launch shape of the parallel line sweep gives the same bits: x-lines
    in CTAs of 32 to 256 threads and (FP32, 256 to 2048 points) the streamed
    kernel; y-lines with 1, 2, 4 or 8 lines per CTA."""
    import torch
    nl = 37
    dt = torch.float64 if precision == "f64" else torch.float32
    fn = lib.cdr_gpu_relax_lines_2d_f64 if precision == "f64" else lib.cdr_gpu_relax_lines_2d_f32
    fp32 = 1 if precision == "f32" else 0
    for direction, (nx, ny) in ((_lib.DIR_X, (n, nl)), (_lib.DIR_Y, (nl, n))):
        # elements per thread: fixed by the line length (y-lines over 1024 points: 16)
        K = 16 if direction == _lib.DIR_Y and n > 1024 else 8
        tpl = 1
        while tpl * K < n:
            tpl *= 2
        so, x, b = make_op(nx, ny, 5), grid(nx, ny, 8), grid(nx, ny, 9)
        sor, _ = (oracle.setup_lines_x if direction == _lib.DIR_X else oracle.setup_lines_y)(so)
        g = sor.copy()
        if fp32:
            g[0][1:-1, 1:-1] = 1.0 / sor[0][1:-1, 1:-1]
        pitch = ((nx + 2 + 31) // 32) * 32
        tpitch = ((ny + 2 + 31) // 32) * 32
        dso, dbb = padded(so, pitch, dt), padded(b, pitch, dt)
        dsor = padded(g, pitch if direction == _lib.DIR_X else tpitch, dt)
        if direction == _lib.DIR_X:
            caps = [32, 64, 128, 256] + ([0] if fp32 and 256 <= n <= 2048 else [])
        else:
            caps = sorted({max(32, tpl * gg) for gg in (1, 2, 4, 8) if tpl * gg <= (1024 if fp32 else 512)})
        outs = []
        for cap in caps:
            _lib.check(lib.cdr_gpu_lines_set_shape(direction, fp32, 5, n, nl, 0, K, cap))
            dx = padded(x, pitch, dt)
            for updown in (0, 1):
                _lib.check(fn(ptr(dso), 5, ptr(dx), ptr(dbb), ptr(dsor), nx, ny, pitch, tpitch, direction, updown, 0,
                              stream()))
            outs.append(host(dx))
        assert lib.cdr_gpu_lines_stream_status(stream()) == 0
        for cap, o in zip(caps[1:], outs[1:]):
            np.testing.assert_array_equal(o, outs[0], err_msg="direction %d cap %d" % (direction, cap))
        xr = x.copy()
        ofn = oracle.relax_lines_x if direction == _lib.DIR_X else oracle.relax_lines_y
        ofn(so, xr, b, sor, 0)
        ofn(so, xr, b, sor, 1)
        assert rel_err(outs[0][:, :nx + 2], xr) < (1e-12 if not fp32 else 2e-4)


def test_pinned_line_shape_is_used(lib):
    """cdr_gpu_lines_set_shape pins a launch shape for a geometry: a solver
    created afterwards (autotuner on) keeps it, and the solve converges; a shape
    that cannot run the lines is refused."""
    import ctypes
    from cedar_b200.solver import Solver2D
    from cedar_b200.config import Config
    n = 383
    so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=4, contrast=100.0, aniso=0.5)
    _lib.check(lib.cdr_gpu_lines_set_shape(_lib.DIR_Y, 1, 5, n, n, 0, 8, 64))
    _lib.check(lib.cdr_gpu_lines_set_shape(_lib.DIR_X, 1, 5, n, n, 0, 8, 0))
    assert lib.cdr_gpu_lines_set_shape(_lib.DIR_Y, 1, 5, 5000, 5000, 0, 4, 64) != 0
    s = Solver2D(so, Config({"solver": {"relaxation": "line-xy", "max-iter": 30, "tol": 1e-9},
                             "gpu": {"precision": "fp32-ir", "autotune": True}}))
    s.solve(b)
    assert s.history[-1] < 1e-9
    for d, want in ((_lib.DIR_Y, (8, 64)), (_lib.DIR_X, (8, 0))):
        K, cap = ctypes.c_int(), ctypes.c_int()
        _lib.check(lib.cdr_gpu_lines_shape(d, 1, 5, n, n, 0, ctypes.byref(K), ctypes.byref(cap)))
        assert (K.value, cap.value) == want


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("nx,ny,ns", [(37, 100, 5), (64, 383, 5), (255, 1024, 3), (96, 2047, 5), (2047, 2047, 5),
                                      (9, 12, 5), (1, 40, 5)])
def test_one_launch_y_sweep_equals_two_launches(lib, precision, nx, ny, ns):
    """y-lines with a sync buffer sweep both colours in one launch (blocks of
    column pairs, a flag between neighbouring blocks): bit-identical to the two
    one-colour launches for every lines-per-CTA shape, both directions of
    sweep; the buffer is left zeroed and no block gives up."""
    import torch
    dt = torch.float64 if precision == "f64" else torch.float32
    fp32 = precision == "f32"
    fn = lib.cdr_gpu_relax_lines_2d_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_f32
    fns = lib.cdr_gpu_relax_lines_2d_sync_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_sync_f32
    from oracle import oracle as O
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 8), grid(nx, ny, 9)
    sy, _ = O.setup_lines_y(so)
    g = sy.copy()
    if fp32:
        g[0][1:-1, 1:-1] = 1.0 / sy[0][1:-1, 1:-1]
    pitch = ((nx + 2 + 31) // 32) * 32
    tpitch = ((ny + 2 + 31) // 32) * 32
    dso, dbb, dsy = padded(so, pitch, dt), padded(b, pitch, dt), padded(g, tpitch, dt)
    words = lib.cdr_gpu_lines_sync_words(nx)
    sync = torch.zeros(words, dtype=torch.int32, device="cuda")
    K = 16 if ny > 1024 else 8
    tpl = 1
    while tpl * K < ny:
        tpl *= 2
    caps = sorted({max(32, tpl * gg) for gg in (1, 2, 4, 8) if tpl * gg <= (1024 if fp32 else 512)})
    for cap in caps:
        _lib.check(lib.cdr_gpu_lines_set_shape(_lib.DIR_Y, 1 if fp32 else 0, ns, ny, nx, 0, K, cap))
        for updown in (0, 1):
            d1, d2 = padded(x, pitch, dt), padded(x, pitch, dt)
            for _ in range(2):
                _lib.check(fn(ptr(dso), ns, ptr(d1), ptr(dbb), ptr(dsy), nx, ny, pitch, tpitch, _lib.DIR_Y, updown, 0,
                              stream()))
                _lib.check(fns(ptr(dso), ns, ptr(d2), ptr(dbb), ptr(dsy), nx, ny, pitch, tpitch, _lib.DIR_Y, updown,
                               16, ptr(sync), stream()))  # CDR_LINES_YPAIR
            np.testing.assert_array_equal(host(d2), host(d1), err_msg="cap %d updown %d" % (cap, updown))
            assert int(sync.abs().sum().item()) == 0
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("nx,ny,ns", [(37, 100, 5), (300, 41, 5), (64, 63, 3), (1023, 255, 5), (96, 2047, 5)])
def test_zero_start_sweep_does_not_read_the_iterate(lib, precision, nx, ny, ns):
    """CDR_LINES_ZERO_START (x zero on entry, its interior not read): a sweep of
    an iterate whose interior holds garbage equals the sweep of a zero iterate,
    x- and y-lines, both sweep directions, the one-launch y sweep, the streamed
    x-line shape, and a pitch the register-chunk kernels cannot take (the sweep
    then clears x itself)."""
    import torch
    dt = torch.float64 if precision == "f64" else torch.float32
    fp32 = precision == "f32"
    fn = lib.cdr_gpu_relax_lines_2d_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_f32
    fns = lib.cdr_gpu_relax_lines_2d_sync_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_sync_f32
    from oracle import oracle as O
    so, junk, b = make_op(nx, ny, ns), grid(nx, ny, 8), grid(nx, ny, 9)
    zero = np.zeros_like(junk)
    sx, _ = O.setup_lines_x(so)
    sy, _ = O.setup_lines_y(so)
    gx, gy = sx.copy(), sy.copy()
    if fp32:
        gx[0][1:-1, 1:-1] = 1.0 / sx[0][1:-1, 1:-1]
        gy[0][1:-1, 1:-1] = 1.0 / sy[0][1:-1, 1:-1]
    sync = torch.zeros(lib.cdr_gpu_lines_sync_words(nx), dtype=torch.int32, device="cuda")
    for pitch in (((nx + 2 + 31) // 32) * 32, nx + 3):
        tpitch = ((ny + 2 + 31) // 32) * 32
        dso, dbb = padded(so, pitch, dt), padded(b, pitch, dt)
        dsx, dsy = padded(gx, pitch, dt), padded(gy, tpitch, dt)
        for direction, fac in ((_lib.DIR_X, dsx), (_lib.DIR_Y, dsy)):
            for updown in (0, 1):
                for extra in ((0, 4) if direction == _lib.DIR_X and fp32 else (0,)):
                    for use_sync in ((False, True) if direction == _lib.DIR_Y else (False,)):
                        d1, d2 = padded(zero, pitch, dt), padded(junk, pitch, dt)
                        if use_sync:  # both colours in one launch (CDR_LINES_YPAIR)
                            _lib.check(fns(ptr(dso), ns, ptr(d1), ptr(dbb), ptr(fac), nx, ny, pitch, tpitch, direction,
                                           updown, extra | 16, ptr(sync), stream()))
                            _lib.check(fns(ptr(dso), ns, ptr(d2), ptr(dbb), ptr(fac), nx, ny, pitch, tpitch, direction,
                                           updown, extra | 24, ptr(sync), stream()))
                        else:
                            _lib.check(fn(ptr(dso), ns, ptr(d1), ptr(dbb), ptr(fac), nx, ny, pitch, tpitch, direction,
                                          updown, extra, stream()))
                            _lib.check(fn(ptr(dso), ns, ptr(d2), ptr(dbb), ptr(fac), nx, ny, pitch, tpitch, direction,
                                          updown, extra | 8, stream()))
                        msg = "pitch %d dir %d updown %d flags %d sync %s" % (pitch, direction, updown, extra, use_sync)
                        np.testing.assert_array_equal(host(d2), host(d1), err_msg=msg)
    assert int(sync.abs().sum().item()) == 0
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("nx,ny,ns", [(37, 100, 5), (64, 63, 3), (255, 1024, 5), (96, 2047, 5), (9, 12, 5)])
def test_packed_y_couplings_sweep_bitwise(lib, precision, nx, ny, ns):
    """cdr_gpu_pack_ylines_2d_* writes line i's couplings after the y factors;
    a y sweep with CDR_LINES_YPACKED reads them there: bit-identical to the
    sweep that reads the operator, both directions of sweep, with and without
    a zero start, over several launch shapes, one launch per colour and both
    colours in one launch."""
    import torch
    dt = torch.float64 if precision == "f64" else torch.float32
    fp32 = precision == "f32"
    fn = lib.cdr_gpu_relax_lines_2d_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_f32
    fns = lib.cdr_gpu_relax_lines_2d_sync_f64 if not fp32 else lib.cdr_gpu_relax_lines_2d_sync_f32
    fp = lib.cdr_gpu_pack_ylines_2d_f64 if not fp32 else lib.cdr_gpu_pack_ylines_2d_f32
    sync = torch.zeros(lib.cdr_gpu_lines_sync_words(nx), dtype=torch.int32, device="cuda")
    from oracle import oracle as O
    so, x, b = make_op(nx, ny, ns), grid(nx, ny, 8), grid(nx, ny, 9)
    sy, _ = O.setup_lines_y(so)
    g = sy.copy()
    if fp32:
        g[0][1:-1, 1:-1] = 1.0 / sy[0][1:-1, 1:-1]
    pitch = ((nx + 2 + 31) // 32) * 32
    tpitch = ((ny + 2 + 31) // 32) * 32
    dso, dbb = padded(so, pitch, dt), padded(b, pitch, dt)
    npk = 6 if ns == 5 else 2
    big = np.zeros((2 + npk, nx + 2, ny + 2))
    big[:2] = g
    dsy = padded(big, tpitch, dt)
    _lib.check(fp(ptr(dso), ns, ptr(dsy), nx, ny, pitch, tpitch, stream()))
    K = 16 if ny > 1024 else 8
    tpl = 1
    while tpl * K < ny:
        tpl *= 2
    caps = sorted({max(32, tpl * gg) for gg in (1, 2, 4, 8) if tpl * gg <= (1024 if fp32 else 512)})
    for cap in caps:
        _lib.check(lib.cdr_gpu_lines_set_shape(_lib.DIR_Y, 1 if fp32 else 0, ns, ny, nx, 0, K, cap))
        for updown in (0, 1):
            for flags in (0, 8):
                d1, d2, d3 = padded(x, pitch, dt), padded(x, pitch, dt), padded(x, pitch, dt)
                for _ in range(2):
                    _lib.check(fn(ptr(dso), ns, ptr(d1), ptr(dbb), ptr(dsy), nx, ny, pitch, tpitch, _lib.DIR_Y, updown,
                                  flags, stream()))
                    _lib.check(fn(ptr(dso), ns, ptr(d2), ptr(dbb), ptr(dsy), nx, ny, pitch, tpitch, _lib.DIR_Y, updown,
                                  flags | 32, stream()))
                    _lib.check(fns(ptr(dso), ns, ptr(d3), ptr(dbb), ptr(dsy), nx, ny, pitch, tpitch, _lib.DIR_Y,
                                   updown, flags | 48, ptr(sync), stream()))  # CDR_LINES_YPAIR | CDR_LINES_YPACKED
                np.testing.assert_array_equal(host(d2), host(d1),
                                              err_msg="cap %d updown %d flags %d" % (cap, updown, flags))
                np.testing.assert_array_equal(host(d3), host(d1),
                                              err_msg="pair: cap %d updown %d flags %d" % (cap, updown, flags))
    assert int(sync.abs().sum().item()) == 0
    assert lib.cdr_gpu_lines_stream_status(stream()) == 0
