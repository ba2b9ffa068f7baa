"""Test-problem operators and right-hand sides (host side, numpy, FP64).

Stencils use Cedar's 2D storage: array ``so[k, j, i]`` of shape ``(k, ny+2, nx+2)``
with one ghost ring, i fastest, planes ``c, w, s`` (five_pt) or ``c, w, s, sw, nw``
(nine_pt).  ``w``/``s``/``sw``/``nw`` hold the negated couplings
``-A[(i,j),(i-1,j)]``, ``-A[(i,j),(i,j-1)]``, ``-A[(i,j),(i-1,j-1)]`` and
``-A[(i-1,j),(i,j-1)]``; Dirichlet-zero boundaries are zero couplings into the
ghost ring.  Indices below are 0-based with the ghost at 0 and n+1, exactly the
C++ indices of the reference's gallery.
"""
import math

import numpy as np

C, W, S, SW, NW = 0, 1, 2, 3, 4


def poisson(nx, ny):
    """5-point Laplacian scaled by h^2, as ``gallery::poisson`` (src/2d/gallery.cc:7-39)."""
    so = np.zeros((3, ny + 2, nx + 2))
    hx = 1.0 / (nx + 1)
    hy = 1.0 / (ny + 1)
    xh = hy / hx
    yh = hx / hy
    so[S, 2:ny + 1, 1:nx + 1] = 1.0 * yh
    so[W, 1:ny + 1, 2:nx + 1] = 1.0 * xh
    so[C, 1:ny + 1, 1:nx + 1] = 2 * xh + 2 * yh
    return so


def diag_diffusion(nx, ny, dx, dy):
    """Anisotropic 5-point operator, as ``gallery::diag_diffusion`` (src/2d/gallery.cc:42-74)."""
    so = np.zeros((3, ny + 2, nx + 2))
    hx = 1.0 / (nx + 1)
    hy = 1.0 / (ny + 1)
    xh = hy / hx
    yh = hx / hy
    so[S, 2:ny + 1, 1:nx + 1] = dy * yh
    so[W, 1:ny + 1, 2:nx + 1] = dx * xh
    so[C, 1:ny + 1, 1:nx + 1] = 2 * dx * xh + 2 * dy * yh
    return so


def fe(nx, ny):
    """Constant 9-point bilinear-FE operator, as ``gallery::fe`` (src/2d/gallery.cc:77-110)."""
    so = np.zeros((5, ny + 2, nx + 2))
    so[S, 2:ny + 1, 1:nx + 1] = 1.0
    so[W, 1:ny + 1, 2:nx + 1] = 1.0
    so[SW, 2:ny + 1, 2:nx + 1] = 1.0
    so[NW, 2:ny + 1, 2:nx + 1] = 1.0
    so[C, 1:ny + 1, 1:nx + 1] = 8.0
    return so


def poisson_rhs_sin2pi(nx, ny):
    """b = 8 pi^2 sin(2 pi x) sin(2 pi y) h^2 at x = i h (examples/basic-2d-ser/poisson.cc:15-37)."""
    b = np.zeros((ny + 2, nx + 2))
    hx = 1.0 / (nx + 1)
    hy = 1.0 / (ny + 1)
    h2 = hx * hy
    pi = math.pi
    i = np.arange(1, nx + 1)
    j = np.arange(1, ny + 1)
    x = i * hx
    y = j * hy
    # same evaluation order as the reference lambda: 8*(pi*pi)*sin(2*pi*x)*sin(2*pi*y), then * h2
    sx = np.sin(2 * pi * x)
    sy = np.sin(2 * pi * y)
    b[1:ny + 1, 1:nx + 1] = ((8 * (pi * pi)) * sx[None, :]) * sy[:, None] * h2
    return b


def poisson_exact_sin2pi(nx, ny):
    """Exact solution sin(2 pi x) sin(2 pi y) on the whole grid including ghosts."""
    hx = 1.0 / (nx + 1)
    hy = 1.0 / (ny + 1)
    pi = math.pi
    x = np.arange(nx + 2) * hx
    y = np.arange(ny + 2) * hy
    return np.sin(2 * pi * x)[None, :] * np.sin(2 * pi * y)[:, None]


# --------------------------------------------------------------------------
# Heterogeneous bilinear (Q1) finite elements.  The reference gallery has only
# constant-coefficient operators; this assembler builds the 9-point operator of
# -div(K grad u) on an (nx+1) x (ny+1) cell mesh of the unit square with
# Dirichlet-zero boundary, K = diag(kx, ky) constant per cell.  Element matrix:
# kx * (K1 (x) M1)' + ky * (M1 (x) K1)' with K1 = [[1,-1],[-1,1]] / h and
# M1 = h/6 [[2,1],[1,2]] (the h factors cancel on a square cell).
# --------------------------------------------------------------------------

def q1_element_matrices():
    """Reference element matrices (Ex, Ey) on a square cell, local nodes
    0:(0,0) 1:(1,0) 2:(0,1) 3:(1,1).  A_e = kx*Ex + ky*Ey."""
    K1 = np.array([[1.0, -1.0], [-1.0, 1.0]])
    M1 = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0
    # node (a, b) with a = x-index, b = y-index; local id = a + 2 b
    Ex = np.zeros((4, 4))
    Ey = np.zeros((4, 4))
    for b1 in range(2):
        for a1 in range(2):
            for b2 in range(2):
                for a2 in range(2):
                    Ex[a1 + 2 * b1, a2 + 2 * b2] = K1[a1, a2] * M1[b1, b2]
                    Ey[a1 + 2 * b1, a2 + 2 * b2] = M1[a1, a2] * K1[b1, b2]
    return Ex, Ey


def fe_hetero(kx, ky):
    """9-point stencil from per-cell coefficients.

    ``kx``, ``ky``: arrays of shape (ny+1, nx+1); cell (cj, ci) has corner nodes
    (ci, cj), (ci+1, cj), (ci, cj+1), (ci+1, cj+1) in the 0-based node index that
    includes the boundary nodes 0 and n+1.  Returns ``so`` of shape (5, ny+2, nx+2).
    """
    kx = np.asarray(kx, dtype=np.float64)
    ky = np.asarray(ky, dtype=np.float64)
    ncy, ncx = kx.shape
    nx, ny = ncx - 1, ncy - 1
    Ex, Ey = q1_element_matrices()
    so = np.zeros((5, ny + 2, nx + 2))
    # entries per cell (cell with SW node (i-1, j-1) and NE node (i, j) = so index (i, j))
    # diagonal: each node gets A_e[l,l] from its 4 cells
    diag = np.zeros((ny + 2, nx + 2))
    for l, (a, b) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        diag[b:b + ncy, a:a + ncx] += kx * Ex[l, l] + ky * Ey[l, l]
    # horizontal edge coupling between (i-1,j) and (i,j): cells below (j-1) and above (j)
    # cell local pair (0,1) for the bottom edge of cell (cj=j) and (2,3) for the top edge of cell (cj=j-1)
    h_bot = kx * Ex[0, 1] + ky * Ey[0, 1]   # nodes (ci,cj)-(ci+1,cj)
    h_top = kx * Ex[2, 3] + ky * Ey[2, 3]   # nodes (ci,cj+1)-(ci+1,cj+1)
    aw = np.zeros((ny + 2, nx + 2))          # A[(i,j),(i-1,j)] stored at (i,j)
    aw[0:ncy, 1:ncx + 1] += h_bot
    aw[1:ncy + 1, 1:ncx + 1] += h_top
    v_left = kx * Ex[0, 2] + ky * Ey[0, 2]  # nodes (ci,cj)-(ci,cj+1)
    v_right = kx * Ex[1, 3] + ky * Ey[1, 3]  # nodes (ci+1,cj)-(ci+1,cj+1)
    as_ = np.zeros((ny + 2, nx + 2))         # A[(i,j),(i,j-1)] stored at (i,j)
    as_[1:ncy + 1, 0:ncx] += v_left
    as_[1:ncy + 1, 1:ncx + 1] += v_right
    d_sw = kx * Ex[0, 3] + ky * Ey[0, 3]     # (ci,cj)-(ci+1,cj+1): stored at NE node
    d_nw = kx * Ex[1, 2] + ky * Ey[1, 2]     # (ci+1,cj)-(ci,cj+1): stored at NE node
    asw = np.zeros((ny + 2, nx + 2))
    anw = np.zeros((ny + 2, nx + 2))
    asw[1:ncy + 1, 1:ncx + 1] = d_sw
    anw[1:ncy + 1, 1:ncx + 1] = d_nw
    so[C, 1:ny + 1, 1:nx + 1] = diag[1:ny + 1, 1:nx + 1]
    # couplings only between interior nodes (Dirichlet: zero into the ghost ring)
    so[W, 1:ny + 1, 2:nx + 1] = -aw[1:ny + 1, 2:nx + 1]
    so[S, 2:ny + 1, 1:nx + 1] = -as_[2:ny + 1, 1:nx + 1]
    so[SW, 2:ny + 1, 2:nx + 1] = -asw[2:ny + 1, 2:nx + 1]
    so[NW, 2:ny + 1, 2:nx + 1] = -anw[2:ny + 1, 2:nx + 1]
    return so


def stencil_to_csr(so):
    """Assemble the full sparse matrix of a 2D stencil (interior unknowns, i fastest)."""
    import scipy.sparse as sp
    nst, JJ, II = so.shape
    nx, ny = II - 2, JJ - 2
    idx = lambda i, j: (j - 1) * nx + (i - 1)
    rows, cols, vals = [], [], []
    I, J = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1))
    I = I.ravel()
    J = J.ravel()
    k = idx(I, J)
    rows.append(k); cols.append(k); vals.append(so[C, J, I])

    def couple(mask, i2, j2, v):
        rows.append(k[mask]); cols.append(idx(i2[mask], j2[mask])); vals.append(-v[mask])

    couple(I > 1, I - 1, J, so[W, J, I])
    couple(I < nx, I + 1, J, so[W, J, I + 1])
    couple(J > 1, I, J - 1, so[S, J, I])
    couple(J < ny, I, J + 1, so[S, J + 1, I])
    if nst == 5:
        couple((I > 1) & (J > 1), I - 1, J - 1, so[SW, J, I])
        couple((I < nx) & (J < ny), I + 1, J + 1, so[SW, J + 1, I + 1])
        couple((I < nx) & (J > 1), I + 1, J - 1, so[NW, J, I + 1])
        couple((I > 1) & (J < ny), I - 1, J + 1, so[NW, J + 1, I])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(nx * ny, nx * ny))
