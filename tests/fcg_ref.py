"""Flexible CG (Notay's FCG(1)) with the oracle's cycle as the preconditioner:
the CPU restatement the GPU's CDR_KRYLOV_FCG solve is checked against.

TEST INFRASTRUCTURE ONLY (imports the oracle)."""
import numpy as np

from cedar_b200 import gallery as G


def fcg(oracle, so, b, relax="line-xy", npre=1, npost=1, tol=1e-10, maxiter=200, num_levels=-1):
    """Returns (x, history of |b - A x_k| / |b - A x_0|, final relative residual).
    The residual is formed from x every iteration, as the GPU solve does.
    num_levels: levels of the oracle's cycle (-1: the reference's rule)."""
    ny, nx = b.shape[0] - 2, b.shape[1] - 2
    A = G.stencil_to_csr(so)
    pre = oracle.Solver(so, relax=relax, maxiter=1, tol=1e-300, nrelax_pre=npre, nrelax_post=npost,
                        num_levels=num_levels)

    def M(r):
        rr = np.zeros_like(b)
        rr[1:-1, 1:-1] = r.reshape(ny, nx)
        z, _ = pre.solve(rr)
        return z[1:-1, 1:-1].ravel()

    bv = b[1:-1, 1:-1].ravel()
    x = np.zeros_like(bv)
    r = bv.copy()
    r0 = np.linalg.norm(r)
    hist = []
    p = q = None
    for _ in range(maxiter):
        z = M(r)
        p = z if p is None else z - (z @ q) / (p @ q) * p
        q = A @ p
        alpha = (p @ r) / (p @ q)
        x += alpha * p
        r = bv - A @ x
        hist.append(np.linalg.norm(r) / r0)
        if hist[-1] < tol:
            break
    xo = np.zeros_like(b)
    xo[1:-1, 1:-1] = x.reshape(ny, nx)
    true_rel = np.linalg.norm(bv - A @ x) / r0
    return xo, np.array(hist), true_rel
