"""The FP32 preconditioner with its fine-level iterate kept in FP64.

With flexible CG around the FP32 cycle (settings.fp64_fine_iterate, the
default), the fine level's interpolate-add widens the iterate to FP64; the
post-smoothing then runs in FP32 on a correction from zero whose right-hand
side is the residual of the FP64 iterate, formed in FP64 arithmetic over the
FP32 operator in difference form (couplings and row-sum excess).  The
preconditioner's output is the FP64 iterate plus the FP32 correction.

Checks, through the C ABI:

* the row-sum excess: c - (sum of the point's couplings) formed in FP64 and
  rounded, bit for bit against numpy;
* the wide residual: bit for bit against the same FP64 sums in numpy, and the
  post-smoothing's initial guess zeroed on the interior;
* the wide interpolate-add: bit for bit against the oracle's FP64
  interpolate-add (BMG2_SymStd_interp_add) run on the FP32 data;
* on heterogeneous problems, the FP32-cycle FCG with the widened iterate needs
  no more iterations than with the FP32 one, its first relative residual (one
  preconditioned step) is far below the FP32 one's, and its solution agrees
  with the FP64-cycle solve.
"""
import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import problems as P
from tests.gpu_util import dev, host, padded, ptr, stream
from tests.test_gpu_kernels import grid, make_op

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    return _lib.load()


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def rowsum_excess(so):
    c, w, s = so[0], so[1], so[2]
    a = w[1:-1, 1:-1] + w[1:-1, 2:] + s[1:-1, 1:-1] + s[2:, 1:-1]
    if so.shape[0] == 5:
        sw, nw = so[3], so[4]
        a = a + sw[1:-1, 1:-1] + sw[2:, 2:] + nw[1:-1, 2:] + nw[2:, 1:-1]
    dg = np.zeros_like(c)
    dg[1:-1, 1:-1] = f32(c[1:-1, 1:-1] - a)
    return dg


def residual_wide(so32, dg, x, b32):
    """b - dg x - sum a (x - x_nb), FP64, in the kernel's order, rounded to FP32."""
    w, s = so32[1], so32[2]
    X = x[1:-1, 1:-1]
    a = b32[1:-1, 1:-1] - dg[1:-1, 1:-1] * X
    a = a - w[1:-1, 1:-1] * (X - x[1:-1, :-2])
    a = a - w[1:-1, 2:] * (X - x[1:-1, 2:])
    a = a - s[1:-1, 1:-1] * (X - x[:-2, 1:-1])
    a = a - s[2:, 1:-1] * (X - x[2:, 1:-1])
    if so32.shape[0] == 5:
        sw, nw = so32[3], so32[4]
        a = a - sw[1:-1, 1:-1] * (X - x[:-2, :-2])
        a = a - nw[1:-1, 2:] * (X - x[:-2, 2:])
        a = a - nw[2:, 1:-1] * (X - x[2:, :-2])
        a = a - sw[2:, 2:] * (X - x[2:, 2:])
    r = np.zeros_like(x)
    r[1:-1, 1:-1] = f32(a)
    return r


@pytest.mark.parametrize("nx,ny,ns", [(37, 100, 5), (255, 127, 3), (2047, 33, 5), (1, 9, 5), (130, 129, 5)])
def test_rowsum_excess_and_wide_residual_bitwise(lib, nx, ny, ns):
    import torch
    so = make_op(nx, ny, ns)
    pitch = ((nx + 2 + 31) // 32) * 32
    dso64 = padded(so, pitch)
    ddg = torch.full((ny + 2, pitch), 7.0, dtype=torch.float32, device="cuda")
    ddg[0, :] = 0; ddg[-1, :] = 0; ddg[:, 0] = 0; ddg[:, nx + 1:] = 0
    _lib.check(lib.cdr_gpu_rowsum_excess_2d(ptr(dso64), ns, ptr(ddg), nx, ny, pitch, stream()))
    dg = rowsum_excess(so)
    np.testing.assert_array_equal(host(ddg)[:, :nx + 2], dg)
    so32 = f32(so)
    x = grid(nx, ny, 3) * 1e3 + 1e5  # a large, smooth-ish part: the difference form's case
    b32 = f32(grid(nx, ny, 4))
    want = residual_wide(so32, dg, x, b32)
    dr = torch.zeros((ny + 2, pitch), dtype=torch.float32, device="cuda")
    dz = torch.ones((ny + 2, pitch), dtype=torch.float32, device="cuda")
    dz[0, :] = 0; dz[-1, :] = 0; dz[:, 0] = 0; dz[:, nx + 1:] = 0
    dso32, dx, db32 = padded(so32, pitch, torch.float32), padded(x, pitch), padded(b32, pitch, torch.float32)
    _lib.check(lib.cdr_gpu_residual_2d_wide(ptr(dso32), ptr(ddg), ns, ptr(dx), ptr(db32), ptr(dr), ptr(dz), nx, ny,
                                            pitch, stream()))
    np.testing.assert_array_equal(host(dr)[:, :nx + 2], want)
    assert float(dz.abs().sum().item()) == 0.0


def test_wide_residual_refuses_unaligned_rows(lib):
    import torch
    t = torch.zeros(8192, dtype=torch.float32, device="cuda")
    t64 = torch.zeros(8192, dtype=torch.float64, device="cuda")
    rc = lib.cdr_gpu_residual_2d_wide(ptr(t), ptr(t), 5, ptr(t64), ptr(t), ptr(t), ptr(t), 30, 30, 33, stream())
    assert rc == 1  # CDR_ERR_ARG: pitch not a multiple of 4


@pytest.mark.parametrize("nx,ny,ns", [(37, 100, 5), (64, 47, 3), (255, 255, 5), (2047, 17, 5)])
def test_wide_interp_add_equals_fp64_interp_on_fp32_data(lib, nx, ny, ns):
    import torch
    from oracle import oracle as O
    O.build()
    so = f32(make_op(nx, ny, ns))
    nxc, nyc = (nx - 1) // 2 + 1, (ny - 1) // 2 + 1
    ci = f32(O.setup_interp(so, nxc, nyc))
    xc, r, x = f32(grid(nxc, nyc, 6)), f32(grid(nx, ny, 5)), f32(grid(nx, ny, 7))
    want = O.interp_add(ci, xc, r.copy(), so, x.copy())
    F = torch.float32
    dci, dxc = dev(ci, F), dev(xc, F)
    # Cedar's pitch (2 x 2 blocks of fine points per thread) and a padded one
    # (the row kernel: 16-byte rows)
    for pitch in (nx + 2, ((nx + 2 + 31) // 32) * 32):
        dout = torch.full((ny + 2, pitch), 3.0, dtype=torch.float64, device="cuda")
        dr, dso, dx = padded(r, pitch, F), padded(so, pitch, F), padded(x, pitch, F)
        _lib.check(lib.cdr_gpu_interp_add_2d_wide(ptr(dci), ptr(dxc), ptr(dr), ptr(dso), ns, ptr(dx), ptr(dout), nx,
                                                  ny, pitch, nxc, nyc, nxc + 2, stream()))
        got = host(dout)
        np.testing.assert_array_equal(got[1:-1, 1:nx + 1], want[1:-1, 1:-1], err_msg="pitch %d" % pitch)


def _fcg(so, b, prec, fine, tol=1e-4, levels=5):
    from cedar_b200.config import Config
    from cedar_b200.solver import Solver2D
    conf = {"solver": {"relaxation": "line-xy", "max-iter": 400, "tol": tol, "num-levels": levels,
                       "cycle": {"nrelax-pre": 1, "nrelax-post": 1}},
            "gpu": {"precision": prec, "krylov": "fcg", "coarse-solve": "inverse", "fcg-replace": 10,
                    "fine-iterate": fine}}
    s = Solver2D(so, Config(conf))
    x = s.solve(b)
    h = s.history.copy()
    s.close()
    return x, h


@pytest.mark.parametrize("n", [511, 1023])
def test_fcg_with_wide_fine_iterate(lib, n):
    so, b = P.hetero_diffusion(n)
    x64, h64 = _fcg(so, b, "fp64", "fp64")
    xw, hw = _fcg(so, b, "fp32-ir", "fp64")
    xn, hn = _fcg(so, b, "fp32-ir", "fp32")
    assert h64[-1] < 1e-4 and hw[-1] < 1e-4 and hn[-1] < 1e-4
    assert len(hw) <= len(hn), (len(hw), len(hn), len(h64))
    # one preconditioned step: the FP32 iterate's rounding shows in the residual
    assert hw[0] < hn[0] / 2, (hw[0], hn[0], h64[0])
    err = np.linalg.norm(xw - x64) / np.linalg.norm(x64)
    assert err < 1e-3, err

