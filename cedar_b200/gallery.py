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


# --------------------------------------------------------------------------
# 3D: trilinear (Q1) finite elements, 27-point operators in Cedar's 14-plane
# lower-half storage (include/cedar/3d/base_types.h:4-20): p, pw, ps, b, psw,
# pnw, bw, bnw, bn, bne, be, bse, bs, bsw.  Plane q at point s holds the negated
# coupling between the two nodes listed in PLANES3[q] (offsets from s).
# --------------------------------------------------------------------------
P3, PW3, PS3, B3, PSW3, PNW3, BW3, BNW3, BN3, BNE3, BE3, BSE3, BS3, BSW3 = range(14)
PLANES3 = {
    PW3: ((0, 0, 0), (-1, 0, 0)), PS3: ((0, 0, 0), (0, -1, 0)), B3: ((0, 0, 0), (0, 0, -1)),
    PSW3: ((0, 0, 0), (-1, -1, 0)), PNW3: ((0, -1, 0), (-1, 0, 0)), BW3: ((0, 0, 0), (-1, 0, -1)),
    BNW3: ((0, -1, 0), (-1, 0, -1)), BN3: ((0, -1, 0), (0, 0, -1)), BNE3: ((-1, -1, 0), (0, 0, -1)),
    BE3: ((-1, 0, 0), (0, 0, -1)), BSE3: ((-1, 0, 0), (0, -1, -1)), BS3: ((0, 0, 0), (0, -1, -1)),
    BSW3: ((0, 0, 0), (-1, -1, -1)),
}


def q1_element_matrices_3d():
    """(Ex, Ey, Ez) on a unit cube, local node l = a + 2b + 4c; A_e = h*k*(Ex+Ey+Ez)."""
    K1 = np.array([[1.0, -1.0], [-1.0, 1.0]])
    M1 = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0
    E = [np.zeros((8, 8)) for _ in range(3)]
    for l1 in range(8):
        a1, b1, c1 = l1 & 1, (l1 >> 1) & 1, l1 >> 2
        for l2 in range(8):
            a2, b2, c2 = l2 & 1, (l2 >> 1) & 1, l2 >> 2
            E[0][l1, l2] = K1[a1, a2] * M1[b1, b2] * M1[c1, c2]
            E[1][l1, l2] = M1[a1, a2] * K1[b1, b2] * M1[c1, c2]
            E[2][l1, l2] = M1[a1, a2] * M1[b1, b2] * K1[c1, c2]
    return E


def fe3_hetero(k):
    """27-point trilinear-FE operator of -div(k grad u), k per cell (nz+1, ny+1, nx+1),
    Dirichlet zero boundary, h = 1/(n+1) per direction (cube cells)."""
    k = np.asarray(k, dtype=np.float64)
    ncz, ncy, ncx = k.shape
    nx, ny, nz = ncx - 1, ncy - 1, ncz - 1
    h = 1.0 / ncx
    Ex, Ey, Ez = q1_element_matrices_3d()
    Ae = h * (Ex + Ey + Ez)
    # coupling arrays C[d][node] = A[node, node + d] for every offset d, ghost-inclusive node index
    shape = (nz + 2, ny + 2, nx + 2)
    C = {}
    for l1 in range(8):
        o1 = (l1 & 1, (l1 >> 1) & 1, l1 >> 2)
        for l2 in range(8):
            o2 = (l2 & 1, (l2 >> 1) & 1, l2 >> 2)
            d = (o2[0] - o1[0], o2[1] - o1[1], o2[2] - o1[2])
            arr = C.setdefault(d, np.zeros(shape))
            arr[o1[2]:o1[2] + ncz, o1[1]:o1[1] + ncy, o1[0]:o1[0] + ncx] += k * Ae[l1, l2]
    so = np.zeros((14,) + shape)
    inner = np.zeros(shape, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    so[P3][inner] = C[(0, 0, 0)][inner]
    for q, (oa, ob) in PLANES3.items():
        d = (ob[0] - oa[0], ob[1] - oa[1], ob[2] - oa[2])
        # plane value at s = -A[s+oa, s+ob] = -C[d][s+oa]; both nodes must be interior
        Z, Y, X = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
        ax, ay, az = X + oa[0], Y + oa[1], Z + oa[2]
        bx, by, bz = X + ob[0], Y + ob[1], Z + ob[2]
        ok = ((ax >= 1) & (ax <= nx) & (ay >= 1) & (ay <= ny) & (az >= 1) & (az <= nz)
              & (bx >= 1) & (bx <= nx) & (by >= 1) & (by <= ny) & (bz >= 1) & (bz <= nz))
        vals = np.zeros(shape)
        vals[ok] = -C[d][az[ok], ay[ok], ax[ok]]
        so[q] = vals
    return so


# --------------------------------------------------------------------------
# 3D seven-point operators (include/cedar/3d/base_types.h seven_pt): 4 planes
# p, pw, ps, b with pw/ps/b at s the negated couplings to s-(1,0,0), s-(0,1,0)
# and s-(0,0,1).
# --------------------------------------------------------------------------

def _seven_pt(nx, ny, nz, cx, cy, cz):
    so = np.zeros((4, nz + 2, ny + 2, nx + 2))
    hx, hy, hz = 1.0 / (nx + 1), 1.0 / (ny + 1), 1.0 / (nz + 1)
    xh = hy * hz / hx
    yh = hx * hz / hy
    zh = hx * hy / hz
    so[PS3, 1:nz + 1, 2:ny + 1, 1:nx + 1] = cy * yh
    so[PW3, 1:nz + 1, 1:ny + 1, 2:nx + 1] = cx * xh
    so[B3, 2:nz + 1, 1:ny + 1, 1:nx + 1] = cz * zh
    so[P3, 1:nz + 1, 1:ny + 1, 1:nx + 1] = 2.0 * cx * xh + 2.0 * cy * yh + 2.0 * cz * zh
    return so


def poisson3(nx, ny, nz):
    """Seven-point Laplacian scaled by h^3/h^2, as ``cdr3::gallery::poisson`` (src/3d/gallery.cc:7-55)."""
    return _seven_pt(nx, ny, nz, 1.0, 1.0, 1.0)  # 2.0*1.0*xh == 2.0*xh exactly


def diag_diffusion3(nx, ny, nz, dx, dy, dz):
    """Anisotropic seven-point operator, as ``cdr3::gallery::diag_diffusion`` (src/3d/gallery.cc:58-107)."""
    return _seven_pt(nx, ny, nz, dx, dy, dz)


def fd3_hetero(k):
    """Seven-point finite-difference operator of -div(k grad u) with k given at
    the grid points (nz+2, ny+2, nx+2), ghosts included: the coupling between
    neighbours a, b is the harmonic mean 2 k_a k_b / (k_a + k_b) times xh, yh or
    zh (the poisson3 scaling), p the sum of a point's six couplings (those into
    the Dirichlet ghost layer included, then dropped from the stored planes)."""
    k = np.asarray(k, dtype=np.float64)
    nz, ny, nx = k.shape[0] - 2, k.shape[1] - 2, k.shape[2] - 2
    hx, hy, hz = 1.0 / (nx + 1), 1.0 / (ny + 1), 1.0 / (nz + 1)
    xh, yh, zh = hy * hz / hx, hx * hz / hy, hx * hy / hz
    hm = lambda a, b: 2.0 * a * b / (a + b)
    so = np.zeros((4,) + k.shape)
    cw = np.zeros(k.shape); cs = np.zeros(k.shape); cb = np.zeros(k.shape)
    cw[:, :, 1:] = hm(k[:, :, 1:], k[:, :, :-1]) * xh   # coupling of s and s-(1,0,0)
    cs[:, 1:, :] = hm(k[:, 1:, :], k[:, :-1, :]) * yh
    cb[1:, :, :] = hm(k[1:, :, :], k[:-1, :, :]) * zh
    I = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    p = np.zeros(k.shape)
    p[I] = cw[I] + cs[I] + cb[I]
    p[1:nz + 1, 1:ny + 1, 1:nx + 1] += (cw[1:nz + 1, 1:ny + 1, 2:nx + 2] + cs[1:nz + 1, 2:ny + 2, 1:nx + 1]
                                        + cb[2:nz + 2, 1:ny + 1, 1:nx + 1])
    so[P3][I] = p[I]
    so[PW3, 1:nz + 1, 1:ny + 1, 2:nx + 1] = cw[1:nz + 1, 1:ny + 1, 2:nx + 1]
    so[PS3, 1:nz + 1, 2:ny + 1, 1:nx + 1] = cs[1:nz + 1, 2:ny + 1, 1:nx + 1]
    so[B3, 2:nz + 1, 1:ny + 1, 1:nx + 1] = cb[2:nz + 1, 1:ny + 1, 1:nx + 1]
    return so


def seven_to_27(so):
    """The 14-plane storage of a seven-point operator (the other couplings zero)."""
    out = np.zeros((14,) + so.shape[1:])
    out[:4] = so
    return out


def poisson3_rhs_sin2pi(nx, ny, nz):
    """b = 12 pi^2 sin(2 pi x) sin(2 pi y) sin(2 pi z) hx hy hz (test/3d/test_poisson.cc:12-41)."""
    hx, hy, hz = 1.0 / (nx + 1), 1.0 / (ny + 1), 1.0 / (nz + 1)
    h2 = hx * hy * hz
    pi = math.pi
    sx = np.sin(2 * pi * (np.arange(1, nx + 1) * hx))
    sy = np.sin(2 * pi * (np.arange(1, ny + 1) * hy))
    sz = np.sin(2 * pi * (np.arange(1, nz + 1) * hz))
    b = np.zeros((nz + 2, ny + 2, nx + 2))
    b[1:-1, 1:-1, 1:-1] = ((12 * (pi * pi)) * sx[None, None, :] * sy[None, :, None]) * sz[:, None, None] * h2
    return b


def poisson3_exact_sin2pi(nx, ny, nz):
    """sin(2 pi x) sin(2 pi y) sin(2 pi z) on the whole grid including ghosts (test_poisson.cc:44-68)."""
    hx, hy, hz = 1.0 / (nx + 1), 1.0 / (ny + 1), 1.0 / (nz + 1)
    pi = math.pi
    sx = np.sin(2 * pi * (np.arange(nx + 2) * hx))
    sy = np.sin(2 * pi * (np.arange(ny + 2) * hy))
    sz = np.sin(2 * pi * (np.arange(nz + 2) * hz))
    return sx[None, None, :] * sy[None, :, None] * sz[:, None, None]


def stencil3_to_csr(so):
    """Full sparse matrix of a 14-plane (or seven-point, 4-plane) 3D stencil
    (interior unknowns, i fastest)."""
    import scipy.sparse as sp
    if so.shape[0] == 4:
        so = seven_to_27(so)
    _, KK, JJ, II = so.shape
    nx, ny, nz = II - 2, JJ - 2, KK - 2
    idx = lambda i, j, k: ((k - 1) * ny + (j - 1)) * nx + (i - 1)
    rows, cols, vals = [], [], []
    Z, Y, X = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
    rows.append(idx(X, Y, Z)); cols.append(idx(X, Y, Z)); vals.append(so[P3, Z, Y, X])
    for q, (oa, ob) in PLANES3.items():
        # entry at s couples s+oa and s+ob; s ranges over all points with both nodes interior
        Zs, Ys, Xs = np.meshgrid(np.arange(KK), np.arange(JJ), np.arange(II), indexing="ij")
        ax, ay, az = Xs + oa[0], Ys + oa[1], Zs + oa[2]
        bx, by, bz = Xs + ob[0], Ys + ob[1], Zs + ob[2]
        ok = ((ax >= 1) & (ax <= nx) & (ay >= 1) & (ay <= ny) & (az >= 1) & (az <= nz)
              & (bx >= 1) & (bx <= nx) & (by >= 1) & (by <= ny) & (bz >= 1) & (bz <= nz))
        v = -so[q][ok]
        r1, r2 = idx(ax[ok], ay[ok], az[ok]), idx(bx[ok], by[ok], bz[ok])
        rows += [r1, r2]; cols += [r2, r1]; vals += [v, v]
    N = nx * ny * nz
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


def periodic_poisson(nx, ny, periodic=(True, False)):
    """5-point Poisson on an nx x ny grid with periodic directions, as the
    reference's periodic example builds it (examples/basic-2d-ser/periodic.cc:16-131):
    a periodic direction has nx (ny) distinct points, h = 1/nx there, the
    coupling to the ghost line enters the operator, and the ghost lines of the
    operator and of b hold copies of the opposite interior lines.  Returns
    (so, b, exact) with b = 8 pi^2 sin(2 pi x) sin(2 pi y) h^2 and
    exact = sin(2 pi x) sin(2 pi y) at the interior points."""
    px, py = bool(periodic[0]), bool(periodic[1])
    l, m = nx, ny
    so = np.zeros((3, ny + 2, nx + 2))
    hx = 1.0 / ((nx - 1 if px else nx) + 1)
    hy = 1.0 / ((ny - 1 if py else ny) + 1)
    xh, yh = hy / hx, hx / hy
    ibeg = 1 if px else 2
    jbeg = 1 if py else 2
    so[S, jbeg:m + 1, 1:l + 1] = 1.0 * yh
    so[W, 1:m + 1, ibeg:l + 1] = 1.0 * xh
    so[C, 1:m + 1, 1:l + 1] = 2 * xh + 2 * yh
    if px:
        so[:, 1:m + 1, 0] = so[:, 1:m + 1, l]
        so[:, 1:m + 1, l + 1] = so[:, 1:m + 1, 1]
    if py:
        so[:, 0, 1:l + 1] = so[:, m, 1:l + 1]
        so[:, m + 1, 1:l + 1] = so[:, 1, 1:l + 1]
    x = np.arange(1, l + 1) * hx
    y = np.arange(1, m + 1) * hy
    b = np.zeros((ny + 2, nx + 2))
    b[1:-1, 1:-1] = 8 * math.pi ** 2 * np.outer(np.sin(2 * math.pi * y), np.sin(2 * math.pi * x)) * (hx * hy)
    if px:
        b[:, 0] = b[:, l]
        b[:, l + 1] = b[:, 1]
    if py:
        b[0, :] = b[m, :]
        b[m + 1, :] = b[1, :]
    exact = np.zeros_like(b)
    exact[1:-1, 1:-1] = np.outer(np.sin(2 * math.pi * y), np.sin(2 * math.pi * x))
    return so, b, exact
