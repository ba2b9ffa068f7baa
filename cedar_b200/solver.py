"""``cdr2::solver`` on the GPU: setup in the constructor, ``solve``/``vcycle`` after.

Mirrors include/cedar/2d/solver.h:45-129 and include/cedar/multilevel.h:80-298:

    so = gallery.poisson(nx, ny)          # stencil_op<five_pt>, Cedar layout
    bmg = Solver2D(so, Config("config.json"))
    x = bmg.solve(b)                      # zeros initial guess, like solve(b)
    bmg.history                           # relative l2 residual per cycle

All arithmetic runs in libcdrgpu.so on the current CUDA device; host arrays
are numpy arrays in Cedar's layout (grid functions (ny+2, nx+2), stencils
(nstencil, ny+2, nx+2)).  Device arrays may be torch CUDA tensors.
"""
import ctypes

import numpy as np

from . import _lib
from .config import Config, MLSettings

PLANE_NAMES = {"so": 0, "x": 1, "b": 2, "res": 3, "sor": 4, "sory": 5, "ci": 6}


def _settings(ms: MLSettings, dim=2):
    if dim == 2 and ms.relaxation.startswith("plane"):
        raise NotImplementedError("relaxation %r is a 3D smoother" % ms.relaxation)
    if dim == 3 and ms.relaxation.startswith("line"):
        raise NotImplementedError("relaxation %r is a 2D smoother (3D: point or plane-*)" % ms.relaxation)
    # solver.cg-solver ("LU", "cedar", "redist") is read by the reference's MPI solvers only
    # (src/2d/mpi/solver.cc:68, include/cedar/3d/mpi/solver.h:212); its serial solvers, which
    # these mirror, always factor the coarsest level (banded Cholesky)
    s = _lib.Settings()
    _lib.check(_lib.load().cdr_gpu_settings_default(ctypes.byref(s)))
    s.relaxation = _lib.RELAX[ms.relaxation]
    s.nrelax_pre = ms.nrelax_pre
    s.nrelax_post = ms.nrelax_post
    s.num_levels = ms.num_levels
    s.maxiter = ms.maxiter
    s.tol = ms.tol
    s.min_coarse = ms.min_coarse
    s.precision = _lib.PREC[ms.precision]
    s.use_graph = 1 if ms.use_graph else 0
    s.line_flags = ((_lib.LINES_EXACT if ms.line_solve == "sequential" else 0) |
                    (0 if ms.autotune else _lib.LINES_NOTUNE) | (_lib.LINES_STREAM if ms.line_stream else 0))
    s.fuse_coarse = ms.fuse_coarse
    if ms.krylov != "none" and dim != 2:
        raise NotImplementedError("gpu.krylov = %r: the Krylov outer iteration is 2D only" % ms.krylov)
    if ms.coarse_solve != "banded" and dim != 2:
        raise NotImplementedError("gpu.coarse-solve = %r is a 2D-solver option" % ms.coarse_solve)
    s.krylov = _lib.KRYLOV[ms.krylov]
    s.coarse_solve = _lib.COARSE[ms.coarse_solve]
    if ms.fp32_levels and dim != 2:
        raise NotImplementedError("gpu.fp32-levels is a 2D-solver option")
    s.fp32_levels = ms.fp32_levels
    s.cycle = 1 if ms.cycle == "f" else 0
    s.krylov_replace = ms.fcg_replace
    if dim == 2 and ms.periodic[2]:
        raise ValueError("grid.periodic: a 2D grid has no z direction")
    s.periodic = ms.per_mask
    s.fp64_fine_iterate = 1 if ms.fine_iterate == "fp64" else 0
    return s


class Solver2D:
    """BoxMG 2D solver whose setup and solve run on the GPU."""

    def __init__(self, so, conf=None, stream=0):
        self.lib = _lib.load()
        so = np.ascontiguousarray(so, dtype=np.float64)
        if so.ndim != 3 or so.shape[0] not in (3, 5):
            raise ValueError("stencil must have shape (3|5, ny+2, nx+2)")
        self.nstencil = so.shape[0]
        self.ny, self.nx = so.shape[1] - 2, so.shape[2] - 2
        self.settings = conf if isinstance(conf, MLSettings) else MLSettings(conf)
        self._s = _settings(self.settings)
        h = ctypes.c_void_p()
        _lib.check(self.lib.cdr_gpu_solver_create_2d(ctypes.byref(self._s), so.ctypes.data, self.nstencil,
                                                     self.nx, self.ny, ctypes.c_void_p(stream), ctypes.byref(h)))
        self.h = h
        self.history = np.zeros(0)
        self.iters = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.cdr_gpu_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nlevels(self):
        return self.lib.cdr_gpu_solver_nlevels(self.h)

    def timings(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.cdr_gpu_solver_timings(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def level_info(self, level, which="so", fp32=False):
        """(device pointer, nx, ny, pitch, tpitch, nstencil) of a level array."""
        p = ctypes.c_void_p()
        vals = [ctypes.c_int() for _ in range(5)]
        wid = PLANE_NAMES[which] + (16 if fp32 else 0) if which != "abd" else 100
        _lib.check(self.lib.cdr_gpu_solver_level(self.h, level, wid, ctypes.byref(p), *[ctypes.byref(v) for v in vals]))
        return (p.value,) + tuple(v.value for v in vals)

    def level_array(self, level, which="so", fp32=False):
        """Host copy of a level array in Cedar's layout (planes, ny+2, nx+2); the
        transposed y-line factors come back as (2, nx+2, ny+2)."""
        p, nx, ny, pitch, tpitch, ns = self.level_info(level, which, fp32)
        wid = PLANE_NAMES[which] + (16 if fp32 else 0)
        planes = {"so": ns, "sor": 2, "ci": 8}.get(which, 1)
        dt = np.float32 if fp32 else np.float64
        if which == "sory":
            buf = np.zeros((2, nx + 2, tpitch), dtype=dt)
        else:
            buf = np.zeros((planes, ny + 2, pitch), dtype=dt)
        _lib.check(self.lib.cdr_gpu_solver_level_get(self.h, level, wid, buf.ctypes.data, buf.nbytes))
        out = buf[..., :ny + 2] if which == "sory" else buf[..., :nx + 2]
        return np.ascontiguousarray(out if planes > 1 or which == "sory" else out[0])

    def solve(self, b, x=None):
        """Solve A x = b from host arrays (Cedar layout); returns x (numpy)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.shape != (self.ny + 2, self.nx + 2):
            raise ValueError("rhs shape %s does not match the grid" % (b.shape,))
        x = np.zeros_like(b) if x is None else np.ascontiguousarray(x, dtype=np.float64).copy()
        hist = np.zeros(max(self.settings.maxiter, 1))
        it = ctypes.c_int()
        _lib.check(self.lib.cdr_gpu_solver_solve(self.h, b.ctypes.data, x.ctypes.data, ctypes.byref(it),
                                                 hist.ctypes.data, len(hist)))
        self.iters = it.value
        self.history = hist[:it.value].copy()
        return x

    def solve_device(self, b_ptr, x_ptr, pitch):
        """Solve with device buffers (e.g. ``tensor.data_ptr()``), x holds the initial guess."""
        hist = np.zeros(max(self.settings.maxiter, 1))
        it = ctypes.c_int()
        _lib.check(self.lib.cdr_gpu_solver_solve_device(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr),
                                                        pitch, ctypes.byref(it), hist.ctypes.data, len(hist)))
        self.iters = it.value
        self.history = hist[:it.value].copy()

    def vcycle_device(self, b_ptr, x_ptr, pitch):
        _lib.check(self.lib.cdr_gpu_solver_vcycle_device(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr), pitch))


class Solver3D:
    """``cdr3::solver`` (include/cedar/3d/solver.h) on the GPU: 27-point
    (xxvii_pt, 14 planes) or seven-point (seven_pt, 4 planes: p, pw, ps, b) fine
    operator in Cedar's layout (planes, nz+2, ny+2, nx+2)."""

    def __init__(self, so, conf=None, stream=0, dims=None, pitch=None, nstencil=14):
        """so: host array (nstencil, nz+2, ny+2, nx+2), or a device pointer (int)
        with dims = (nx, ny, nz), the row pitch of the device array and nstencil."""
        self.lib = _lib.load()
        self.settings = conf if isinstance(conf, MLSettings) else MLSettings(conf)
        self._s = _settings(self.settings, dim=3)
        h = ctypes.c_void_p()
        if dims is not None:
            self.nx, self.ny, self.nz = dims
            self.nstencil = nstencil
            _lib.check(self.lib.cdr_gpu_solver3_create_device(ctypes.byref(self._s), ctypes.c_void_p(so), nstencil,
                                                              self.nx, self.ny, self.nz, pitch,
                                                              ctypes.c_void_p(stream), ctypes.byref(h)))
        else:
            so = np.ascontiguousarray(so, dtype=np.float64)
            if so.ndim != 4 or so.shape[0] not in (4, 14):
                raise ValueError("stencil must have shape (14 or 4, nz+2, ny+2, nx+2)")
            self.nstencil = so.shape[0]
            self.nz, self.ny, self.nx = so.shape[1] - 2, so.shape[2] - 2, so.shape[3] - 2
            _lib.check(self.lib.cdr_gpu_solver3_create(ctypes.byref(self._s), so.ctypes.data, self.nstencil, self.nx,
                                                       self.ny, self.nz, ctypes.c_void_p(stream), ctypes.byref(h)))
        self.h = h
        self.history = np.zeros(0)
        self.iters = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.cdr_gpu_solver3_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nlevels(self):
        return self.lib.cdr_gpu_solver3_nlevels(self.h)

    def timings(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.cdr_gpu_solver3_timings(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def level_info(self, level, which="so", fp32=False):
        """(device pointer, nx, ny, nz, pitch) of a level array."""
        p = ctypes.c_void_p()
        vals = [ctypes.c_int() for _ in range(4)]
        wid = PLANE_NAMES[which] + (16 if fp32 else 0) if which != "abd" else 100
        _lib.check(self.lib.cdr_gpu_solver3_level(self.h, level, wid, ctypes.byref(p), *[ctypes.byref(v) for v in vals]))
        return (p.value,) + tuple(v.value for v in vals)

    def level_array(self, level, which="so", fp32=False):
        """Host copy of a level array in Cedar's layout (planes, nz+2, ny+2, nx+2)."""
        p, nx, ny, nz, pitch = self.level_info(level, which, fp32)
        wid = PLANE_NAMES[which] + (16 if fp32 else 0)
        planes = {"so": self.nstencil if level == 0 else 14, "ci": 26}.get(which, 1)
        dt = np.float32 if fp32 else np.float64
        buf = np.zeros((planes, nz + 2, ny + 2, pitch), dtype=dt)
        _lib.check(self.lib.cdr_gpu_solver3_level_get(self.h, level, wid, buf.ctypes.data, buf.nbytes))
        out = np.ascontiguousarray(buf[..., :nx + 2])
        return out if planes > 1 else out[0]

    def solve(self, b, x=None):
        """Solve A x = b from host arrays (Cedar layout (nz+2, ny+2, nx+2)); returns x."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.shape != (self.nz + 2, self.ny + 2, self.nx + 2):
            raise ValueError("rhs shape %s does not match the grid" % (b.shape,))
        x = np.zeros_like(b) if x is None else np.ascontiguousarray(x, dtype=np.float64).copy()
        hist = np.zeros(max(self.settings.maxiter, 1))
        it = ctypes.c_int()
        _lib.check(self.lib.cdr_gpu_solver3_solve(self.h, b.ctypes.data, x.ctypes.data, ctypes.byref(it),
                                                  hist.ctypes.data, len(hist)))
        self.iters = it.value
        self.history = hist[:it.value].copy()
        return x

    def solve_device(self, b_ptr, x_ptr, pitch):
        hist = np.zeros(max(self.settings.maxiter, 1))
        it = ctypes.c_int()
        _lib.check(self.lib.cdr_gpu_solver3_solve_device(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr),
                                                         pitch, ctypes.byref(it), hist.ctypes.data, len(hist)))
        self.iters = it.value
        self.history = hist[:it.value].copy()


class BatchSolver2D:
    """A batch of independent 2D problems of one grid size, solved together on
    the GPU (each with its own stopping test, as ``cdr2::solver::solve``).

    ``so_ptr``: device pointer to nb fine operators back to back (each
    nstencil planes of ``pitch*(ny+2)`` doubles)."""

    def __init__(self, so_ptr, nstencil, nx, ny, pitch, nb, conf=None, stream=0):
        self.lib = _lib.load()
        self.settings = conf if isinstance(conf, MLSettings) else MLSettings(conf)
        self._s = _settings(self.settings)
        self.nx, self.ny, self.pitch, self.nb = nx, ny, pitch, nb
        h = ctypes.c_void_p()
        _lib.check(self.lib.cdr_gpu_batch2d_create(ctypes.byref(self._s), ctypes.c_void_p(so_ptr), nstencil, nx, ny,
                                                   pitch, nb, ctypes.c_void_p(stream), ctypes.byref(h)))
        self.h = h
        self.iters = np.zeros(nb, dtype=np.int32)
        self.rel = np.zeros(nb)
        self.done_ms = np.zeros(nb, dtype=np.float32)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cdr_gpu_batch2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nlevels(self):
        return self.lib.cdr_gpu_batch2d_nlevels(self.h)

    def timings(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.cdr_gpu_batch2d_timings(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def solve_device(self, b_ptr, x_ptr, pitch=None):
        """Solve every problem; x (device, nb grids back to back) holds the initial guesses."""
        _lib.check(self.lib.cdr_gpu_batch2d_solve_device(
            self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr), pitch or self.pitch,
            self.iters.ctypes.data, self.rel.ctypes.data, self.done_ms.ctypes.data))


class MixedBatchSolver2D:
    """Independent 2D problems of several grid sizes solved together on the GPU
    (each with its own hierarchy and stopping test, as ``cdr2::solver``): every
    level of every problem with the same grid size shares one FP32 array, so
    one launch of each V-cycle step covers that level of all problems.

    ``classes``: a list of (so_ptr, nstencil, nx, ny, pitch, nb), so_ptr a
    device pointer to nb fine operators back to back.  FP32 cycles with FP64
    refinement (``gpu.precision = "fp32-ir"``)."""

    def __init__(self, classes, conf=None, stream=0):
        self.lib = _lib.load()
        self.settings = conf if isinstance(conf, MLSettings) else MLSettings(conf)
        self._s = _settings(self.settings)
        k = len(classes)
        P = ctypes.c_void_p * k
        I = ctypes.c_int * k
        self.classes = list(classes)
        self._so = P(*[ctypes.c_void_p(c[0]) for c in classes])
        self._ns, self._nx, self._ny = I(*[c[1] for c in classes]), I(*[c[2] for c in classes]), I(*[c[3] for c in classes])
        self._pitch, self._nb = I(*[c[4] for c in classes]), I(*[c[5] for c in classes])
        self.total = sum(c[5] for c in classes)
        h = ctypes.c_void_p()
        _lib.check(self.lib.cdr_gpu_batchmix_create(ctypes.byref(self._s), k, self._so, self._ns, self._nx, self._ny,
                                                    self._pitch, self._nb, ctypes.c_void_p(stream), ctypes.byref(h)))
        self.h = h
        self.iters = np.zeros(self.total, dtype=np.int32)
        self.rel = np.zeros(self.total)
        self.done_ms = np.zeros(self.total, dtype=np.float32)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cdr_gpu_batchmix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nsizes(self):
        return self.lib.cdr_gpu_batchmix_sizes(self.h)

    @property
    def cycle_launches(self):
        return int(self.lib.cdr_gpu_batchmix_cycle_launches(self.h))

    def timings(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.cdr_gpu_batchmix_timings(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def solve_device(self, b_ptrs, x_ptrs):
        """Solve every problem: b_ptrs[c] / x_ptrs[c] (device) hold class c's right-hand sides and initial
        guesses back to back at the class's pitch.  iters, rel, done_ms: per problem, classes in order."""
        k = len(self.classes)
        P = ctypes.c_void_p * k
        bp = P(*[ctypes.c_void_p(p) for p in b_ptrs])
        xp = P(*[ctypes.c_void_p(p) for p in x_ptrs])
        _lib.check(self.lib.cdr_gpu_batchmix_solve_device(self.h, bp, xp, self._pitch, self.iters.ctypes.data,
                                                          self.rel.ctypes.data, self.done_ms.ctypes.data))
