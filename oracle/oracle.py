"""ctypes wrapper of the CPU parity oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py``.  The product path (``cedar_b200``) never imports it.

Array convention (same as the reference, Fortran order with one ghost ring):
a grid function is a numpy array of shape ``(ny+2, nx+2)`` (C order, so i is
fastest) and a stencil with ``k`` planes has shape ``(k, ny+2, nx+2)``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

RELAX = {"point": 0, "line-x": 1, "line-y": 2, "line-xy": 3}
ARR = {"so": 0, "x": 1, "b": 2, "res": 3, "sor0": 4, "sor1": 5, "ci": 6, "abd": 7}
DOWN, UP = 0, 1


class Settings(ctypes.Structure):
    """Mirror of ``ml_settings`` (include/cedar/multilevel_settings.h:28-50)."""
    _fields_ = [("relax", ctypes.c_int), ("nrelax_pre", ctypes.c_int),
                ("nrelax_post", ctypes.c_int), ("num_levels", ctypes.c_int),
                ("maxiter", ctypes.c_int), ("tol", ctypes.c_double),
                ("min_coarse", ctypes.c_int), ("cycle", ctypes.c_int), ("bc", ctypes.c_int)]


def build():
    """Compile ``liboracle.so`` from the C restatement (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(variant=""):
    """variant "" is the reference-faithful build; "fma" contracts a*b+c into FMAs."""
    if variant not in _LIBS:
        path = os.path.join(_HERE, "liboracle%s.so" % ("_" + variant if variant else ""))
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        sig = {
            "o_dpttrf": (I, [I, P, P]),
            "o_dpttrs": (None, [I, P, P, P]),
            "o_dpbtrf_u": (I, [I, I, P, I]),
            "o_dpbtrs_u": (None, [I, I, P, I, P]),
            "o2_residual": (None, [P, P, P, P, I, I, I]),
            "o2_setup_recip": (None, [P, P, I, I]),
            "o2_relax_gs": (None, [P, P, P, P, I, I, I, I]),
            "o2_setup_lines_x": (I, [P, P, I, I]),
            "o2_setup_lines_y": (I, [P, P, I, I]),
            "o2_relax_lines_x": (None, [P, P, P, P, I, I, I, I]),
            "o2_relax_lines_y": (None, [P, P, P, P, I, I, I, I]),
            "o2_restrict": (None, [P, P, P, I, I, I, I]),
            "o2_interp_add": (None, [P, P, P, P, P, I, I, I, I]),
            "o2_setup_interp": (None, [P, P, I, I, I, I, I]),
            "o2_setup_galerkin": (None, [P, P, P, I, I, I, I, I]),
            "o2_setup_cg": (I, [P, I, I, I, P, I]),
            "o2_solve_cg": (None, [P, P, I, I, P, P, I]),
            "o2_l2norm": (D, [P, I, I]),
            "o2_inf_norm": (D, [P, I, I]),
            "o2_num_levels": (I, [I, I, I]),
            "o2_create": (P, [ctypes.POINTER(Settings), P, I, I, I]),
            "o2_destroy": (None, [P]),
            "o2_vcycle": (None, [P, P, P]),
            "o2_cycle": (None, [P, P, P]),
            "o2_solve": (I, [P, P, P, P, I]),
            "o2_solve_fcg": (I, [P, P, P, I, P, I]),
            "o2_bc_code": (I, [I]),
            "o2_relax_gs_per": (None, [P, P, P, P, I, I, I, I, I]),
            "o2_restrict_per": (None, [P, P, P, I, I, I, I, I]),
            "o2_interp_add_per": (None, [P, P, P, P, P, I, I, I, I, I]),
            "o2_setup_interp_per": (None, [P, P, I, I, I, I, I, I]),
            "o2_setup_galerkin_per": (None, [P, P, P, I, I, I, I, I, I]),
            "o2_setup_cg_per": (I, [P, I, I, I, P, I]),
            "o2_solve_cg_per": (None, [P, P, I, I, P, P, I]),
            "o_dpotf2_u": (I, [I, P, I]),
            "o_dpotrs_u": (None, [I, P, I, P]),
            "o_set_threads": (None, [I]),
            "o2_nlevels": (I, [P]),
            "o_num_threads": (I, []),
            "o2_info": (I, [P, I]),
            "o2_level_dims": (None, [P, P]),
            "o2_level_array": (ctypes.POINTER(ctypes.c_double), [P, I, I]),
            "o2_abd_dims": (None, [P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIBS[variant] = L
    return _LIBS[variant]


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


def _dims(so_or_gf):
    return so_or_gf.shape[-1], so_or_gf.shape[-2]  # II, JJ


# ----------------------------------------------------------------- kernels
def residual(so, x, b):
    II, JJ = _dims(x)
    r = np.zeros_like(x)
    lib().o2_residual(_p(so), _p(b), _p(x), _p(r), II, JJ, 1 if so.shape[0] == 3 else 0)
    return r


def setup_recip(so):
    II, JJ = _dims(so)
    sor = np.zeros((2, JJ, II))
    lib().o2_setup_recip(_p(so), _p(sor), II, JJ)
    return sor


def relax_gs(so, x, b, sor, updown):
    II, JJ = _dims(x)
    lib().o2_relax_gs(_p(so), _p(b), _p(x), _p(sor), II, JJ, 1 if so.shape[0] == 3 else 0, updown)
    return x


def setup_lines_x(so):
    II, JJ = _dims(so)
    sor = np.zeros((2, JJ, II))
    info = lib().o2_setup_lines_x(_p(so), _p(sor), II, JJ)
    return sor, info


def setup_lines_y(so):
    """Returns SOR stored transposed, shape (2, II, JJ) (Fortran SOR(JJ,II,2))."""
    II, JJ = _dims(so)
    sor = np.zeros((2, II, JJ))
    info = lib().o2_setup_lines_y(_p(so), _p(sor), II, JJ)
    return sor, info


def relax_lines_x(so, x, b, sor, updown):
    II, JJ = _dims(x)
    lib().o2_relax_lines_x(_p(so), _p(b), _p(x), _p(sor), II, JJ, 1 if so.shape[0] == 3 else 0, updown)
    return x


def relax_lines_y(so, x, b, sor, updown):
    II, JJ = _dims(x)
    lib().o2_relax_lines_y(_p(so), _p(b), _p(x), _p(sor), II, JJ, 1 if so.shape[0] == 3 else 0, updown)
    return x


def restrict(ci, r_fine):
    IIF, JJF = _dims(r_fine)
    IIC, JJC = _dims(ci)
    bc = np.zeros((JJC, IIC))
    lib().o2_restrict(_p(ci), _p(r_fine), _p(bc), IIF, JJF, IIC, JJC)
    return bc


def interp_add(ci, xc, res, so_fine, x):
    """x += P xc + res/c at fine-only points; ``res`` is divided in place (as the reference)."""
    IIC, JJC = _dims(ci)
    IIF, JJF = _dims(x)
    ko = np.ascontiguousarray(so_fine[0])
    lib().o2_interp_add(_p(x), _p(xc), _p(res), _p(ko), _p(ci), IIC, JJC, IIF, JJF)
    return x


def setup_interp(so_fine, nxc, nyc):
    IIF, JJF = _dims(so_fine)
    ci = np.zeros((8, nyc + 2, nxc + 2))
    lib().o2_setup_interp(_p(so_fine), _p(ci), IIF, JJF, nxc + 2, nyc + 2, 1 if so_fine.shape[0] == 3 else 0)
    return ci


def galerkin(so_fine, ci):
    IIF, JJF = _dims(so_fine)
    IIC, JJC = _dims(ci)
    soc = np.zeros((5, JJC, IIC))
    lib().o2_setup_galerkin(_p(so_fine), _p(soc), _p(ci), IIF, JJF, IIC, JJC, 1 if so_fine.shape[0] == 3 else 0)
    return soc


def setup_cg(so):
    II, JJ = _dims(so)
    nx, ny = II - 2, JJ - 2
    abd = np.zeros((nx * ny, nx + 2))  # Fortran ABD(nx+2, nx*ny)
    info = lib().o2_setup_cg(_p(so), II, JJ, so.shape[0], _p(abd), nx + 2)
    return abd, info


def solve_cg(abd, b):
    II, JJ = _dims(b)
    x = np.zeros_like(b)
    bbd = np.zeros((II - 2) * (JJ - 2))
    lib().o2_solve_cg(_p(x), _p(b), II, JJ, _p(abd), _p(bbd), abd.shape[1])
    return x


# ---- periodic branches (cdr2_periodic.c); ipn = o2_bc_code(mask): x -> 2, y -> 1, both -> 3
def bc_code(periodic):
    return lib().o2_bc_code((1 if periodic[0] else 0) | (2 if periodic[1] else 0))


def relax_gs_per(so, x, b, sor, updown, ipn):
    II, JJ = _dims(x)
    lib().o2_relax_gs_per(_p(so), _p(b), _p(x), _p(sor), II, JJ, 1 if so.shape[0] == 3 else 0, updown, ipn)
    return x


def restrict_per(ci, r_fine, ipn):
    """Restriction; the fine vector's ghosts are refreshed in place first (as the reference)."""
    IIF, JJF = _dims(r_fine)
    IIC, JJC = _dims(ci)
    bc = np.zeros((JJC, IIC))
    lib().o2_restrict_per(_p(ci), _p(r_fine), _p(bc), IIF, JJF, IIC, JJC, ipn)
    return bc


def interp_add_per(ci, xc, res, so_fine, x, ipn):
    IIC, JJC = _dims(ci)
    IIF, JJF = _dims(x)
    ko = np.ascontiguousarray(so_fine[0])
    lib().o2_interp_add_per(_p(x), _p(xc), _p(res), _p(ko), _p(ci), IIC, JJC, IIF, JJF, ipn)
    return x


def setup_interp_per(so_fine, nxc, nyc, ipn):
    IIF, JJF = _dims(so_fine)
    ci = np.zeros((8, nyc + 2, nxc + 2))
    lib().o2_setup_interp_per(_p(so_fine), _p(ci), IIF, JJF, nxc + 2, nyc + 2, 1 if so_fine.shape[0] == 3 else 0,
                              ipn)
    return ci


def galerkin_per(so_fine, ci, ipn):
    IIF, JJF = _dims(so_fine)
    IIC, JJC = _dims(ci)
    soc = np.zeros((5, JJC, IIC))
    lib().o2_setup_galerkin_per(_p(so_fine), _p(soc), _p(ci), IIF, JJF, IIC, JJC, 1 if so_fine.shape[0] == 3 else 0,
                                ipn)
    return soc


def setup_cg_per(so, ipn):
    """Dense upper Cholesky factor, column-major (N, N) with N = nx*ny (returned as its transpose in C order)."""
    II, JJ = _dims(so)
    n = (II - 2) * (JJ - 2)
    abd = np.zeros((n, n))
    info = lib().o2_setup_cg_per(_p(so), II, JJ, so.shape[0], _p(abd), ipn)
    return abd, info


def solve_cg_per(abd, b, ipn):
    II, JJ = _dims(b)
    x = np.zeros_like(b)
    bbd = np.zeros((II - 2) * (JJ - 2))
    lib().o2_solve_cg_per(_p(x), _p(b), II, JJ, _p(abd), _p(bbd), ipn)
    return x


def l2norm(r):
    II, JJ = _dims(r)
    return lib().o2_l2norm(_p(r), II, JJ)


def inf_norm(r):
    II, JJ = _dims(r)
    return lib().o2_inf_norm(_p(r), II, JJ)


def dpttrf(d, e):
    d = np.array(d, dtype=np.float64)
    e = np.array(e, dtype=np.float64)
    info = lib().o_dpttrf(len(d), _p(d), _p(e))
    return d, e, info


def dpttrs(d, e, b):
    b = np.array(b, dtype=np.float64)
    lib().o_dpttrs(len(d), _p(np.ascontiguousarray(d)), _p(np.ascontiguousarray(e)), _p(b))
    return b


def dpbtrf_u(ab_fortran, kd):
    """``ab_fortran``: (ldab, n) band matrix in LAPACK upper storage."""
    ab = np.ascontiguousarray(np.asarray(ab_fortran, dtype=np.float64).T)  # column-major
    ldab, n = ab_fortran.shape
    info = lib().o_dpbtrf_u(n, kd, _p(ab), ldab)
    return ab.T.copy(), info


def dpbtrs_u(ab_fortran, kd, b):
    ab = np.ascontiguousarray(np.asarray(ab_fortran, dtype=np.float64).T)
    ldab, n = ab_fortran.shape
    x = np.array(b, dtype=np.float64)
    lib().o_dpbtrs_u(n, kd, _p(ab), ldab, _p(x))
    return x


def num_levels(nx, ny, min_coarse=3):
    return lib().o2_num_levels(nx, ny, min_coarse)


# ------------------------------------------------------------------ solver
def set_threads(n):
    """Host threads of the following oracle calls (0: the environment's count)."""
    lib().o_set_threads(int(n))


def num_threads():
    """Host threads the oracle's cycle kernels use (ORACLE_THREADS / OMP_NUM_THREADS / online CPUs)."""
    return lib().o_num_threads()


class Solver:
    """Serial BoxMG solver: setup in the constructor, as ``cdr2::solver``."""

    def __init__(self, so, relax="point", nrelax_pre=2, nrelax_post=1, num_levels=-1,
                 maxiter=10, tol=1e-8, min_coarse=3, variant="", cycle="v", periodic=(False, False)):
        self.L = lib(variant)
        so = np.ascontiguousarray(so, dtype=np.float64)
        self.nstncl = so.shape[0]
        self.ny, self.nx = so.shape[1] - 2, so.shape[2] - 2
        mask = (1 if periodic[0] else 0) | (2 if periodic[1] else 0)
        self.settings = Settings(RELAX[relax], nrelax_pre, nrelax_post, num_levels, maxiter, tol, min_coarse,
                                 {"v": 0, "f": 1}[cycle], self.L.o2_bc_code(mask))
        self._so = so
        self.h = self.L.o2_create(ctypes.byref(self.settings), _p(so), self.nstncl, self.nx, self.ny)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.o2_destroy(self.h)
            self.h = None

    @property
    def nlevels(self):
        return self.L.o2_nlevels(self.h)

    def info(self):
        return self.L.o2_info(self.h, 0), self.L.o2_info(self.h, 1)

    def level_dims(self, l):
        d = (ctypes.c_int * 3)()
        self.L.o2_level_dims(self.h, l, d)
        return d[0], d[1], d[2]

    def level_array(self, l, which):
        """Copy of a level array in numpy layout."""
        nx, ny, ns = self.level_dims(l)
        II, JJ = nx + 2, ny + 2
        ptr = self.L.o2_level_array(self.h, l, ARR[which])
        if which == "abd":
            d = (ctypes.c_int * 2)()
            self.L.o2_abd_dims(self.h, d)
            n = d[0] * d[1]
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy().reshape(d[1], d[0])
        shape = {"so": (ns, JJ, II), "ci": (8, JJ, II), "sor0": (2, JJ, II),
                 "sor1": (2, II, JJ)}.get(which, (JJ, II))
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy().reshape(shape)

    def vcycle(self, x, b):
        self.L.o2_vcycle(self.h, _p(x), _p(b))
        return x

    def solve(self, b, x=None):
        """Returns (x, history of relative l2 residuals)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if x is None:
            x = np.zeros_like(b)
        hist = np.zeros(max(self.settings.maxiter, 1))
        n = self.L.o2_solve(self.h, _p(b), _p(x), _p(hist), len(hist))
        return x, hist[:n].copy()

    def solve_fcg(self, b, x=None, replace=1):
        """Flexible CG preconditioned by one cycle, to the settings' tol and
        maxiter; the residual is formed every `replace` iterations and to
        confirm convergence.  Returns (x, history)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if x is None:
            x = np.zeros_like(b)
        hist = np.zeros(max(self.settings.maxiter, 1))
        n = self.L.o2_solve_fcg(self.h, _p(b), _p(x), int(replace), _p(hist), len(hist))
        return x, hist[:n].copy()


# ======================================================================= 3D
# Arrays: grid functions (nz+2, ny+2, nx+2); stencils (14, nz+2, ny+2, nx+2);
# interpolation (26, nzc+2, nyc+2, nxc+2).

class Settings3(ctypes.Structure):
    _fields_ = [("nrelax_pre", ctypes.c_int), ("nrelax_post", ctypes.c_int), ("num_levels", ctypes.c_int),
                ("maxiter", ctypes.c_int), ("tol", ctypes.c_double), ("min_coarse", ctypes.c_int),
                ("relax", ctypes.c_int), ("cycle", ctypes.c_int)]


RELAX3 = {"point": 0, "plane-xy": 4, "plane-xz": 5, "plane-yz": 6, "plane-xyz": 7}
PLANE_DIRS = {"xy": 0, "xz": 1, "yz": 2}


_SIG3 = None


def lib3(variant=""):
    global _SIG3
    L = lib(variant)
    if not getattr(L, "_sig3", False):
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        sig = {
            "o3_residual": (None, [P, P, P, P, I, I, I]),
            "o3_setup_recip": (None, [P, P, I, I, I]),
            "o3_relax_gs": (None, [P, P, P, P, I, I, I, I]),
            "o3_restrict": (None, [P, P, P, I, I, I, I, I, I]),
            "o3_interp_add": (None, [P, P, P, P, P, I, I, I, I, I, I]),
            "o3_setup_interp": (None, [P, P, I, I, I, I, I, I]),
            "o3_galerkin": (None, [P, P, P, I, I, I, I, I, I]),
            "o3_setup_cg": (I, [P, I, I, I, P, I]),
            "o3_solve_cg": (None, [P, P, I, I, I, P, P, I]),
            "o3_l2norm": (D, [P, I, I, I]),
            "o3_num_levels": (I, [I, I, I, I]),
            "o3_create": (P, [ctypes.POINTER(Settings3), P, I, I, I, I]),
            "o3_residual7": (None, [P, P, P, P, I, I, I]),
            "o3_relax_gs7": (None, [P, P, P, P, I, I, I, I]),
            "o3_setup_interp7": (None, [P, P, I, I, I, I, I, I]),
            "o3_destroy": (None, [P]),
            "o3_vcycle": (None, [P, P, P]),
            "o3_cycle": (None, [P, P, P]),
            "o3_solve": (I, [P, P, P, P, I]),
            "o3_nlevels": (I, [P]),
            "o3_cg_info": (I, [P]),
            "o3_level_dims": (None, [P, P]),
            "o3_level_array": (ctypes.POINTER(ctypes.c_double), [P, I, I]),
            "o3_relax_planes": (None, [P, I, I, P, P, I]),
            "o3_plane_op": (ctypes.POINTER(ctypes.c_double), [P, I, I, I, ctypes.POINTER(I), ctypes.POINTER(I)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L._sig3 = True
    return L


def _d3(a):
    return a.shape[-1], a.shape[-2], a.shape[-3]


def residual3(so, x, b):
    """27-point (14 planes) or 7-point (4 planes: p, pw, ps, b) residual."""
    II, JJ, KK = _d3(x)
    r = np.zeros_like(x)
    f = lib3().o3_residual7 if so.shape[0] == 4 else lib3().o3_residual
    f(_p(so), _p(b), _p(x), _p(r), II, JJ, KK)
    return r


def setup_recip3(so):
    II, JJ, KK = _d3(so)
    sor = np.zeros(so.shape[1:])
    lib3().o3_setup_recip(_p(so), _p(sor), II, JJ, KK)
    return sor


def relax_gs3(so, x, b, sor, updown):
    II, JJ, KK = _d3(x)
    f = lib3().o3_relax_gs7 if so.shape[0] == 4 else lib3().o3_relax_gs
    f(_p(so), _p(b), _p(x), _p(sor), II, JJ, KK, updown)
    return x


def setup_interp3(so, nxc, nyc, nzc):
    II, JJ, KK = _d3(so)
    ci = np.zeros((26, nzc + 2, nyc + 2, nxc + 2))
    f = lib3().o3_setup_interp7 if so.shape[0] == 4 else lib3().o3_setup_interp
    f(_p(so), _p(ci), II, JJ, KK, nxc + 2, nyc + 2, nzc + 2)
    return ci


def _pad14(so):
    """A seven-point operator (4 planes) in the 14-plane storage, other couplings 0:
    the Galerkin product and the coarse factor read all 14 planes."""
    if so.shape[0] == 14:
        return so
    out = np.zeros((14,) + so.shape[1:])
    out[:so.shape[0]] = so
    return out


def galerkin3(so, ci):
    so = _pad14(so)
    II, JJ, KK = _d3(so)
    IIC, JJC, KKC = _d3(ci)
    soc = np.zeros((14, KKC, JJC, IIC))
    lib3().o3_galerkin(_p(so), _p(soc), _p(ci), II, JJ, KK, IIC, JJC, KKC)
    return soc


def restrict3(ci, r):
    II, JJ, KK = _d3(r)
    IIC, JJC, KKC = _d3(ci)
    bc = np.zeros((KKC, JJC, IIC))
    lib3().o3_restrict(_p(ci), _p(r), _p(bc), II, JJ, KK, IIC, JJC, KKC)
    return bc


def interp_add3(ci, xc, res, so, x):
    IIC, JJC, KKC = _d3(ci)
    II, JJ, KK = _d3(x)
    kp = np.ascontiguousarray(so[0])
    lib3().o3_interp_add(_p(x), _p(xc), _p(res), _p(kp), _p(ci), IIC, JJC, KKC, II, JJ, KK)
    return x


def setup_cg3(so):
    so = _pad14(so)
    II, JJ, KK = _d3(so)
    nx, ny, nz = II - 2, JJ - 2, KK - 2
    nabd1 = nx * (ny + 1) + 2
    abd = np.zeros((nx * ny * nz, nabd1))
    info = lib3().o3_setup_cg(_p(so), II, JJ, KK, _p(abd), nabd1)
    return abd, info


def solve_cg3(abd, b):
    II, JJ, KK = _d3(b)
    x = np.zeros_like(b)
    bbd = np.zeros((II - 2) * (JJ - 2) * (KK - 2))
    lib3().o3_solve_cg(_p(x), _p(b), II, JJ, KK, _p(abd), _p(bbd), abd.shape[1])
    return x


def l2norm3(r):
    II, JJ, KK = _d3(r)
    return lib3().o3_l2norm(_p(r), II, JJ, KK)


class Solver3:
    """Serial 3D BoxMG (27-point or seven-point fine operator; point or plane relaxation)."""

    def __init__(self, so, nrelax_pre=2, nrelax_post=1, num_levels=-1, maxiter=10, tol=1e-8, min_coarse=3,
                 relax="point", cycle="v"):
        self.L = lib3()
        so = np.ascontiguousarray(so, dtype=np.float64)
        assert so.shape[0] in (4, 14)
        self.nz, self.ny, self.nx = so.shape[1] - 2, so.shape[2] - 2, so.shape[3] - 2
        self.s = Settings3(nrelax_pre, nrelax_post, num_levels, maxiter, tol, min_coarse, RELAX3[relax],
                           1 if cycle == "f" else 0)
        self._so = so
        self.h = self.L.o3_create(ctypes.byref(self.s), _p(so), so.shape[0], self.nx, self.ny, self.nz)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.o3_destroy(self.h)
            self.h = None

    @property
    def nlevels(self):
        return self.L.o3_nlevels(self.h)

    def level_dims(self, l):
        d = (ctypes.c_int * 3)()
        self.L.o3_level_dims(self.h, l, d)
        return d[0], d[1], d[2]

    def level_array(self, l, which):
        nx, ny, nz = self.level_dims(l)
        planes = {"so": 14, "ci": 26}.get(which, 1)
        shape = (planes, nz + 2, ny + 2, nx + 2)
        ptr = self.L.o3_level_array(self.h, l, {"so": 0, "x": 1, "b": 2, "res": 3, "sor": 4, "ci": 6}[which])
        a = np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).copy().reshape(shape)
        return a if planes > 1 else a[0]

    def solve(self, b, x=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x is None else x
        hist = np.zeros(max(self.s.maxiter, 1))
        n = self.L.o3_solve(self.h, _p(b), _p(x), _p(hist), len(hist))
        return x, hist[:n].copy()

    def vcycle(self, x, b):
        """One V-cycle from x (in place)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.o3_vcycle(self.h, _p(x), _p(b))
        return x

    def relax_planes(self, level, direction, x, b, updown):
        """One red-black plane sweep (direction 'xy', 'xz' or 'yz') on level arrays x, b (in place)."""
        assert x.flags.c_contiguous and x.dtype == np.float64
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.L.o3_relax_planes(self.h, level, PLANE_DIRS[direction], _p(x), _p(b), updown)
        return x

    def plane_op(self, level, direction, ipl):
        """The 2D nine-point operator (5, n2+2, n1+2) of plane ipl (1-based)."""
        n1, n2 = ctypes.c_int(), ctypes.c_int()
        ptr = self.L.o3_plane_op(self.h, level, PLANE_DIRS[direction], ipl, ctypes.byref(n1), ctypes.byref(n2))
        shape = (5, n2.value + 2, n1.value + 2)
        return np.ctypeslib.as_array(ptr, shape=(int(np.prod(shape)),)).copy().reshape(shape)
