"""Differentiable diffusion solve: implicit differentiation through the BoxMG solver.

``solve_diffusion(kx, ky, f)`` returns u with A(kx, ky) u = f, where A is the
bilinear-FE operator of -div(diag(kx, ky) grad u) on the unit square with
Dirichlet zero boundary (cells (ny+1, nx+1), nodes (ny+2, nx+2) with ghosts).
Forward: the operator is assembled on the device (``cdr_gpu_fe_assemble_2d_f64``),
the BoxMG hierarchy is set up on the device and the system is solved (by default
FP32 V-cycles inside FP64 refinement).  Backward: one adjoint solve
A lam = dL/du on the same (symmetric) hierarchy, then the hand-written kernel
``cdr_gpu_fe_grad_2d_f64`` forms dL/dkx_e = -lam_e^T Ex u_e and
dL/dky_e = -lam_e^T Ey u_e per cell; dL/df = lam.  No cycle intermediate is
stored: this is implicit differentiation of the converged solve.

All tensors are float64 CUDA tensors; a log-coefficient parameter is mapped to
k = exp(theta) by ordinary torch operations around the call.
"""
import ctypes

import torch

from . import _lib
from .config import Config, MLSettings
from .solver import _settings


class _Pool:
    """Reusable device hierarchies, keyed by grid size and settings."""

    def __init__(self):
        self.free = {}

    def acquire(self, nx, ny, key, so_ptr, pitch, stream):
        lst = self.free.setdefault((nx, ny, key), [])
        lib = _lib.load()
        if lst:
            h = lst.pop()
            _lib.check(lib.cdr_gpu_solver_resetup_device(h, ctypes.c_void_p(so_ptr), pitch))
            return h
        s = _settings(MLSettings(Config(_conf_dict(key))))
        h = ctypes.c_void_p()
        _lib.check(lib.cdr_gpu_solver_create_2d_device(ctypes.byref(s), ctypes.c_void_p(so_ptr), 5, nx, ny, pitch,
                                                       ctypes.c_void_p(stream), ctypes.byref(h)))
        return h

    def release(self, nx, ny, key, h):
        self.free.setdefault((nx, ny, key), []).append(h)


_POOL = _Pool()


def _conf_key(tol, maxiter, precision, relaxation):
    return (("solver", (("relaxation", relaxation), ("tol", tol), ("max-iter", maxiter))),
            ("gpu", (("precision", precision),)))


def _conf_dict(key):
    return {k: dict(v) for k, v in key}


def _pitch(n):
    return ((n + 2 + 31) // 32) * 32


def _padded(t, pitch):
    out = torch.zeros((t.shape[0], pitch), dtype=torch.float64, device=t.device)
    out[:, :t.shape[1]] = t
    return out


def _ready():
    """The library's solvers run on their own streams when handed torch's
    default stream: torch's pending writes to the inputs finish first."""
    torch.cuda.current_stream().synchronize()


def _solve(h, b_pad, pitch, maxiter):
    lib = _lib.load()
    x = torch.zeros_like(b_pad)
    _ready()
    it = ctypes.c_int()
    hist = (ctypes.c_double * max(maxiter, 1))()
    _lib.check(lib.cdr_gpu_solver_solve_device(h, ctypes.c_void_p(b_pad.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                               pitch, ctypes.byref(it), hist, max(maxiter, 1)))
    return x, it.value, hist[it.value - 1] if it.value else float("nan")


class DiffusionSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, kx, ky, f, tol, maxiter, precision, relaxation):
        lib = _lib.load()
        ncy, ncx = kx.shape
        nx, ny = ncx - 1, ncy - 1
        if f.shape != (ny + 2, nx + 2):
            raise ValueError("rhs must have shape (ny+2, nx+2) = %s" % ((ny + 2, nx + 2),))
        kx = kx.detach().to(torch.float64).contiguous()
        ky = ky.detach().to(torch.float64).contiguous()
        stream = torch.cuda.current_stream().cuda_stream
        pitch = _pitch(nx)
        so = torch.empty((5, ny + 2, pitch), dtype=torch.float64, device=kx.device)
        _lib.check(lib.cdr_gpu_fe_assemble_2d_f64(ctypes.c_void_p(kx.data_ptr()), ctypes.c_void_p(ky.data_ptr()),
                                                  ncx, ctypes.c_void_p(so.data_ptr()), nx, ny, pitch,
                                                  ctypes.c_void_p(stream)))
        key = _conf_key(tol, maxiter, precision, relaxation)
        _ready()
        h = _POOL.acquire(nx, ny, key, so.data_ptr(), pitch, stream)
        b = _padded(f.detach().to(torch.float64), pitch)
        u, iters, rel = _solve(h, b, pitch, maxiter)
        ctx.info = {"iterations": iters, "final_rel_resid": rel}
        needs = any(ctx.needs_input_grad[:3])
        if needs:
            ctx.save_for_backward(u)
            ctx.solver = h
            ctx.geom = (nx, ny, pitch, key, maxiter)
        else:
            _POOL.release(nx, ny, key, h)
        return u[:, :nx + 2].contiguous()

    @staticmethod
    def backward(ctx, grad_u):
        lib = _lib.load()
        (u,) = ctx.saved_tensors
        nx, ny, pitch, key, maxiter = ctx.geom
        h = ctx.solver
        g = _padded(grad_u.detach().to(torch.float64), pitch)
        g[0, :] = 0.0
        g[-1, :] = 0.0
        g[:, 0] = 0.0
        g[:, nx + 1:] = 0.0
        if float(g.abs().max()) == 0.0:
            lam = torch.zeros_like(g)
        else:
            lam, _, _ = _solve(h, g, pitch, maxiter)  # A symmetric: adjoint = same hierarchy
        gkx = torch.empty((ny + 1, nx + 1), dtype=torch.float64, device=u.device)
        gky = torch.empty_like(gkx)
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.cdr_gpu_fe_grad_2d_f64(ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(lam.data_ptr()), nx, ny,
                                              pitch, ctypes.c_void_p(gkx.data_ptr()), ctypes.c_void_p(gky.data_ptr()),
                                              nx + 1, ctypes.c_void_p(stream)))
        _POOL.release(nx, ny, key, h)
        ctx.solver = None
        return gkx, gky, lam[:, :nx + 2].contiguous(), None, None, None, None


def solve_diffusion(kx, ky, f, tol=1e-10, maxiter=60, precision="fp32-ir", relaxation="line-xy"):
    """u = A(kx, ky)^{-1} f, differentiable in kx, ky and f."""
    return DiffusionSolve.apply(kx, ky, f, tol, maxiter, precision, relaxation)


def solve_log_diffusion(theta, f, **kw):
    """Isotropic k = exp(theta) per cell (theta may be an FP32 parameter)."""
    k = torch.exp(theta.to(torch.float64))
    return solve_diffusion(k, k, f, **kw)


class _BatchPool:
    """Reusable batch hierarchies (cdr_gpu_batch2d), keyed by batch size, grid
    size and settings; a reused batch is set up again on the new operators."""

    def __init__(self):
        self.free = {}

    def acquire(self, nb, nx, ny, key, so_ptr, pitch, stream):
        lst = self.free.setdefault((nb, nx, ny, key), [])
        lib = _lib.load()
        if lst:
            h = lst.pop()
            _lib.check(lib.cdr_gpu_batch2d_resetup_device(h, ctypes.c_void_p(so_ptr), pitch))
            return h
        s = _settings(MLSettings(Config(_conf_dict(key))))
        h = ctypes.c_void_p()
        _lib.check(lib.cdr_gpu_batch2d_create(ctypes.byref(s), ctypes.c_void_p(so_ptr), 5, nx, ny, pitch, nb,
                                              ctypes.c_void_p(stream), ctypes.byref(h)))
        return h

    def release(self, nb, nx, ny, key, h):
        self.free.setdefault((nb, nx, ny, key), []).append(h)


_BPOOL = _BatchPool()


def _solve_batch(h, b_pad, pitch, nb):
    """Every problem of the batch from a zero guess: (x, per-problem cycles, relative residuals)."""
    import numpy as np
    lib = _lib.load()
    x = torch.zeros_like(b_pad)
    iters = np.zeros(nb, dtype=np.int32)
    _ready()
    rel = np.zeros(nb)
    _lib.check(lib.cdr_gpu_batch2d_solve_device(h, ctypes.c_void_p(b_pad.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                                pitch, iters.ctypes.data, rel.ctypes.data, None))
    return x, iters, rel


class BatchDiffusionSolve(torch.autograd.Function):
    """DiffusionSolve for B independent problems of one size at once: the B
    operators are assembled, set up and solved as one batch (each problem with
    its own stopping test), and backward runs the B adjoint solves as one batch
    on the same hierarchies, then the gradient kernel per problem."""

    @staticmethod
    def forward(ctx, kx, ky, f, tol, maxiter, precision, relaxation):
        lib = _lib.load()
        nb, ncy, ncx = kx.shape
        nx, ny = ncx - 1, ncy - 1
        if f.shape != (nb, ny + 2, nx + 2):
            raise ValueError("rhs must have shape (B, ny+2, nx+2) = %s" % ((nb, ny + 2, nx + 2),))
        kx = kx.detach().to(torch.float64).contiguous()
        ky = ky.detach().to(torch.float64).contiguous()
        stream = torch.cuda.current_stream().cuda_stream
        pitch = _pitch(nx)
        so = torch.empty((nb, 5, ny + 2, pitch), dtype=torch.float64, device=kx.device)
        for p in range(nb):
            _lib.check(lib.cdr_gpu_fe_assemble_2d_f64(ctypes.c_void_p(kx[p].data_ptr()),
                                                      ctypes.c_void_p(ky[p].data_ptr()), ncx,
                                                      ctypes.c_void_p(so[p].data_ptr()), nx, ny, pitch,
                                                      ctypes.c_void_p(stream)))
        key = _conf_key(tol, maxiter, precision, relaxation)
        _ready()
        h = _BPOOL.acquire(nb, nx, ny, key, so.data_ptr(), pitch, stream)
        b = torch.zeros((nb, ny + 2, pitch), dtype=torch.float64, device=kx.device)
        b[:, :, :nx + 2] = f.detach().to(torch.float64)
        u, iters, rel = _solve_batch(h, b, pitch, nb)
        ctx.info = {"iterations": iters, "final_rel_resid": rel}
        if any(ctx.needs_input_grad[:3]):
            ctx.save_for_backward(u)
            ctx.solver = h
            ctx.geom = (nb, nx, ny, pitch, key)
        else:
            _BPOOL.release(nb, nx, ny, key, h)
        return u[:, :, :nx + 2].contiguous()

    @staticmethod
    def backward(ctx, grad_u):
        lib = _lib.load()
        (u,) = ctx.saved_tensors
        nb, nx, ny, pitch, key = ctx.geom
        h = ctx.solver
        g = torch.zeros((nb, ny + 2, pitch), dtype=torch.float64, device=u.device)
        g[:, 1:ny + 1, 1:nx + 1] = grad_u.detach().to(torch.float64)[:, 1:ny + 1, 1:nx + 1]
        lam, _, _ = _solve_batch(h, g, pitch, nb)  # A symmetric: adjoint = same hierarchies
        gkx = torch.empty((nb, ny + 1, nx + 1), dtype=torch.float64, device=u.device)
        gky = torch.empty_like(gkx)
        stream = torch.cuda.current_stream().cuda_stream
        for p in range(nb):
            _lib.check(lib.cdr_gpu_fe_grad_2d_f64(ctypes.c_void_p(u[p].data_ptr()), ctypes.c_void_p(lam[p].data_ptr()),
                                                  nx, ny, pitch, ctypes.c_void_p(gkx[p].data_ptr()),
                                                  ctypes.c_void_p(gky[p].data_ptr()), nx + 1,
                                                  ctypes.c_void_p(stream)))
        _BPOOL.release(nb, nx, ny, key, h)
        ctx.solver = None
        return gkx, gky, lam[:, :, :nx + 2].contiguous(), None, None, None, None


def solve_diffusion_batch(kx, ky, f, tol=1e-10, maxiter=60, precision="fp32-ir", relaxation="line-xy"):
    """u[p] = A(kx[p], ky[p])^{-1} f[p] for a batch of B problems of one size
    (kx, ky: (B, ny+1, nx+1) cells; f: (B, ny+2, nx+2)), differentiable in kx, ky and f."""
    return BatchDiffusionSolve.apply(kx, ky, f, tol, maxiter, precision, relaxation)


def solve_log_diffusion_batch(theta, f, **kw):
    """Isotropic k = exp(theta) per cell for a batch (theta: (B, ny+1, nx+1), may be FP32)."""
    k = torch.exp(theta.to(torch.float64))
    return solve_diffusion_batch(k, k, f, **kw)
