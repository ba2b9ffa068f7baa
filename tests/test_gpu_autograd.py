"""Implicit differentiation through the GPU BoxMG solve (hot-path form 2).

Checks: the device FE assembly equals the host assembler bit for bit; the
coefficient-gradient kernel equals its formula; the autograd gradient of
0.5*||u - u_obs||^2 w.r.t. log-coefficients matches central finite differences
(h = 1e-4 on 32 seeded cells) and the gradient built from FP64 CPU-oracle
solves, both within 1e-6 relative."""
import ctypes

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import gallery as G
from cedar_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from cedar_b200 import build
    build.build()
    return _lib.load()


def _grad_formula(kx, ky, u, lam):
    Ex, Ey = G.q1_element_matrices()
    ny1, nx1 = kx.shape
    gx = np.zeros_like(kx)
    gy = np.zeros_like(ky)
    for l1 in range(4):
        for l2 in range(4):
            a1, b1, a2, b2 = l1 & 1, l1 >> 1, l2 & 1, l2 >> 1
            L = lam[b1:b1 + ny1, a1:a1 + nx1]
            U = u[b2:b2 + ny1, a2:a2 + nx1]
            gx -= Ex[l1, l2] * L * U
            gy -= Ey[l1, l2] * L * U
    return gx, gy


@pytest.mark.parametrize("nx,ny", [(15, 15), (20, 13), (63, 64)])
def test_fe_assembly_and_gradient_kernels(lib, nx, ny):
    import torch
    rng = np.random.default_rng(nx + ny)
    kx = np.exp(rng.normal(size=(ny + 1, nx + 1)))
    ky = np.exp(rng.normal(size=(ny + 1, nx + 1)))
    so_ref = G.fe_hetero(kx, ky)
    pitch = ((nx + 2 + 31) // 32) * 32
    dkx, dky = torch.from_numpy(kx).cuda(), torch.from_numpy(ky).cuda()
    so = torch.zeros((5, ny + 2, pitch), dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.cdr_gpu_fe_assemble_2d_f64(ctypes.c_void_p(dkx.data_ptr()), ctypes.c_void_p(dky.data_ptr()),
                                              nx + 1, ctypes.c_void_p(so.data_ptr()), nx, ny, pitch, st))
    np.testing.assert_array_equal(so.cpu().numpy()[:, :, :nx + 2], so_ref)
    u = np.zeros((ny + 2, nx + 2)); u[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    lam = np.zeros((ny + 2, nx + 2)); lam[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    du = torch.zeros((ny + 2, pitch), dtype=torch.float64, device="cuda"); du[:, :nx + 2] = torch.from_numpy(u).cuda()
    dl = torch.zeros_like(du); dl[:, :nx + 2] = torch.from_numpy(lam).cuda()
    gx = torch.zeros_like(dkx); gy = torch.zeros_like(dky)
    _lib.check(lib.cdr_gpu_fe_grad_2d_f64(ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dl.data_ptr()), nx, ny,
                                          pitch, ctypes.c_void_p(gx.data_ptr()), ctypes.c_void_p(gy.data_ptr()),
                                          nx + 1, st))
    rx, ry = _grad_formula(kx, ky, u, lam)
    np.testing.assert_allclose(gx.cpu().numpy(), rx, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(gy.cpu().numpy(), ry, rtol=1e-13, atol=1e-13)
    # gradient identity: d(lam^T A u)/dk_e equals -(our kernel)
    A = G.stencil_to_csr(so_ref)
    val = lam[1:-1, 1:-1].ravel() @ (A @ u[1:-1, 1:-1].ravel())
    h = 1e-6
    cj, ci = 3, 4
    kx2 = kx.copy(); kx2[cj, ci] += h
    val2 = lam[1:-1, 1:-1].ravel() @ (G.stencil_to_csr(G.fe_hetero(kx2, ky)) @ u[1:-1, 1:-1].ravel())
    assert abs((val2 - val) / h + rx[cj, ci]) < 1e-6 * max(1.0, abs(rx[cj, ci]))


def _loss_and_grad(theta_np, f_np, uobs, precision, tol=1e-12):
    import torch
    from cedar_b200.autograd import solve_log_diffusion
    theta = torch.tensor(theta_np, dtype=torch.float64, device="cuda", requires_grad=True)
    f = torch.from_numpy(f_np).cuda()
    u = solve_log_diffusion(theta, f, tol=tol, maxiter=80, precision=precision)
    loss = 0.5 * ((u - uobs) ** 2).sum()
    loss.backward()
    return float(loss.detach()), theta.grad.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp32-ir", "fp64"])
def test_adjoint_gradient_matches_finite_differences_and_oracle(oracle, precision):
    import torch
    n = 63
    theta, theta_obs, f = P.inverse_problem(n)
    from cedar_b200.autograd import solve_log_diffusion
    uobs = solve_log_diffusion(torch.from_numpy(theta_obs).cuda(), torch.from_numpy(f).cuda(), tol=1e-12,
                               maxiter=80, precision="fp64").detach()
    L0, g = _loss_and_grad(theta, f, uobs, precision)
    cells = P.fd_cells(n)
    h = 1e-4
    fd = []
    for cj, ci in cells:
        tp = theta.copy(); tp[cj, ci] += h
        tm = theta.copy(); tm[cj, ci] -= h
        Lp, _ = _loss_and_grad(tp, f, uobs, precision)
        Lm, _ = _loss_and_grad(tm, f, uobs, precision)
        fd.append((Lp - Lm) / (2 * h))
    fd = np.array(fd)
    ga = np.array([g[cj, ci] for cj, ci in cells])
    assert np.linalg.norm(ga - fd) <= 1e-6 * np.linalg.norm(fd), (ga, fd)
    # gradient from FP64 CPU-oracle solves (forward and adjoint) and the element formula
    k = np.exp(theta)
    so = G.fe_hetero(k, k)
    o = oracle.Solver(so, relax="line-xy", maxiter=80, tol=1e-13)
    u, _ = o.solve(f)
    r = u - uobs.cpu().numpy()
    r[0, :] = r[-1, :] = 0.0; r[:, 0] = r[:, -1] = 0.0
    lam, _ = o.solve(np.ascontiguousarray(r))
    gx, gy = _grad_formula(k, k, u, lam)
    g_or = (gx + gy) * k
    assert np.linalg.norm(g - g_or) <= 1e-6 * np.linalg.norm(g_or)


@pytest.mark.parametrize("n,nb", [(63, 3), (127, 2)])
def test_batched_forward_and_adjoint_match_single_problems(lib, n, nb):
    """The batch form (one batched forward solve, one batched adjoint solve,
    the gradient kernel per problem) gives every problem the loss and the
    log-coefficient gradient of its own single-problem solve, to 1e-6
    relative (both solves converge to 1e-10; the FP32 cycles of a batch and of
    a single problem round differently)."""
    import torch
    from cedar_b200.autograd import solve_log_diffusion, solve_log_diffusion_batch
    thetas, fs, uos = [], [], []
    for p in range(nb):
        theta, theta_obs, f = P.inverse_problem(n, seed_theta=8 + 100 * p, seed_src=9 + 100 * p,
                                                seed_obs=10 + 100 * p)
        thetas.append(torch.tensor(theta, dtype=torch.float32, device="cuda"))
        fs.append(torch.from_numpy(f).cuda())
        uos.append(solve_log_diffusion(torch.from_numpy(theta_obs).cuda(), fs[-1], tol=1e-10, maxiter=80).detach())
    th_b = torch.stack(thetas).clone().requires_grad_(True)
    u_b = solve_log_diffusion_batch(th_b, torch.stack(fs), tol=1e-10, maxiter=80)
    loss_b = 0.5 * ((u_b - torch.stack(uos)) ** 2).sum(dim=(1, 2))
    loss_b.sum().backward()
    for p in range(nb):
        th = thetas[p].clone().requires_grad_(True)
        u = solve_log_diffusion(th, fs[p], tol=1e-10, maxiter=80)
        loss = 0.5 * ((u - uos[p]) ** 2).sum()
        loss.backward()
        assert abs(float(loss_b[p].detach()) - float(loss.detach())) <= 1e-6 * abs(float(loss.detach()))
        g, gb = th.grad.double().cpu().numpy(), th_b.grad[p].double().cpu().numpy()
        assert np.abs(gb - g).max() <= 1e-6 * np.abs(g).max(), p
