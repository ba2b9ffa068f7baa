"""Cedar's JSON configuration (``cedar::config``, include/cedar/config.h:12-110).

``get(path, default)`` reads a dotted path such as ``"solver.cycle.nrelax-pre"``.
Keys and defaults are those of ``ml_settings::init`` (src/multilevel_settings.cc:15-61);
note that the reference reads ``solver.min_coarse`` (underscore), so the
``"min-coarse"`` key found in its example configs has no effect there or here.
``solver.cg-solver`` is validated as there but, as in the reference's serial
solvers, does not change the coarsest-level solve (only its MPI solvers read it).
GPU options live under the ``"gpu"`` object: ``precision`` ("fp64" | "fp32-ir"),
``graph`` (bool), ``fuse-coarse`` (levels with both edges at most this many
points run as one fused kernel; 0 = off; default 32), ``line-solve`` ("scan": parallel line substitutions, the
default; "sequential": DPTTRS order, bit-identical to the reference), ``autotune`` (bool, default true: time
the line kernels' launch shapes per level at setup, once per shape and process), ``line-stream`` (bool,
default false: x-line sweeps of 256-2048 points by the persistent kernel whose rows arrive in shared memory
by bulk copies; the autotuner also considers it), ``krylov`` ("none": the
reference's outer loop, the default; "fcg": the cycle preconditions flexible conjugate gradients, 2D only),
``fcg-replace`` (FCG forms the residual b - A x every this many iterations and updates it as r - alpha A p in
between; 1, the default: every iteration),
``coarse-solve`` ("banded": the reference's DPBTRS, the default; "inverse": the setup forms the coarsest
operator's inverse and every cycle multiplies by it, 2D only — for a coarsest level of thousands of unknowns)
``fp32-levels`` (the FP32 cycle keeps this many finest levels in FP32, the rest in FP64; 0 = all, 2D only)
and ``fine-iterate`` ("fp64", the default: with "fcg" and line relaxation the FP32 cycle keeps the fine level's
iterate in FP64 from the interpolate-add on, FP64 arithmetic over its FP32 operator data, so that the
preconditioner's output carries no FP32 rounding of the iterate; "fp32": FP32 throughout).
"""
import json
import os


class Config:
    def __init__(self, src=None):
        if src is None:
            self.tree = {}
        elif isinstance(src, dict):
            self.tree = src
        elif isinstance(src, str) and os.path.exists(src):
            with open(src) as f:
                self.tree = json.load(f)
        elif isinstance(src, str) and src == "":
            self.tree = {}  # config("") is an empty in-memory config (src/config.cc:11-17)
        else:
            raise FileNotFoundError(src)

    def get(self, path, default=None):
        node = self.tree
        for part in path.split("."):
            if not isinstance(node, dict) or part not in node:
                return default
            node = node[part]
        return node

    def getconf(self, path):
        sub = self.get(path)
        return Config(sub) if isinstance(sub, dict) else None

    def getvec(self, path):
        return list(self.get(path, []))


RELAX_NAMES = ["point", "line-x", "line-y", "line-xy", "plane-xy", "plane-xz", "plane-yz", "plane-xyz"]


class MLSettings:
    """``ml_settings`` (include/cedar/multilevel_settings.h:28-50)."""

    def __init__(self, conf=None):
        conf = conf if isinstance(conf, Config) else Config(conf)
        self.relaxation = conf.get("solver.relaxation", "point")
        if self.relaxation not in RELAX_NAMES:
            raise ValueError("invalid relaxation type: %s" % self.relaxation)
        self.cycle = conf.get("solver.cycle.type", "v")
        if self.cycle not in ("v", "f"):
            raise ValueError("invalid cycle type: %s" % self.cycle)
        self.nrelax_pre = int(conf.get("solver.cycle.nrelax-pre", 2))
        self.nrelax_post = int(conf.get("solver.cycle.nrelax-post", 1))
        self.num_levels = int(conf.get("solver.num-levels", -1))
        self.maxiter = int(conf.get("solver.max-iter", 10))
        self.tol = float(conf.get("solver.tol", 1e-8))
        self.min_coarse = int(conf.get("solver.min_coarse", 3))
        self.coarse_solver = conf.get("solver.cg-solver", "LU")
        if self.coarse_solver not in ("LU", "cedar", "redist"):
            raise ValueError("invalid value for solver.cg-solver")
        self.precision = conf.get("gpu.precision", "fp64")
        if self.precision not in ("fp64", "fp32-ir"):
            raise ValueError("invalid gpu.precision: %s" % self.precision)
        self.use_graph = bool(conf.get("gpu.graph", True))
        self.line_solve = conf.get("gpu.line-solve", "scan")
        if self.line_solve not in ("scan", "sequential"):
            raise ValueError("invalid gpu.line-solve: %s" % self.line_solve)
        self.fuse_coarse = int(conf.get("gpu.fuse-coarse", 32))
        if self.fuse_coarse < 0:
            raise ValueError("invalid gpu.fuse-coarse: %d" % self.fuse_coarse)
        self.autotune = bool(conf.get("gpu.autotune", True))
        self.line_stream = bool(conf.get("gpu.line-stream", False))
        self.krylov = conf.get("gpu.krylov", "none")
        if self.krylov not in ("none", "fcg"):
            raise ValueError("invalid gpu.krylov: %s" % self.krylov)
        self.fp32_levels = int(conf.get("gpu.fp32-levels", 0))
        if self.fp32_levels < 0:
            raise ValueError("invalid gpu.fp32-levels: %d" % self.fp32_levels)
        self.fcg_replace = int(conf.get("gpu.fcg-replace", 1))
        if self.fcg_replace < 0:
            raise ValueError("invalid gpu.fcg-replace: %d" % self.fcg_replace)
        self.fine_iterate = conf.get("gpu.fine-iterate", "fp64")
        if self.fine_iterate not in ("fp64", "fp32"):
            raise ValueError("invalid gpu.fine-iterate: %s" % self.fine_iterate)
        self.coarse_solve = conf.get("gpu.coarse-solve", "banded")
        if self.coarse_solve not in ("banded", "inverse"):
            raise ValueError("invalid gpu.coarse-solve: %s" % self.coarse_solve)
        # kernel_params::periodic from grid.periodic (src/kernel_params.cc:72-74)
        pers = list(conf.get("grid.periodic", [False, False, False]))
        self.periodic = tuple(bool(pers[i]) if i < len(pers) else False for i in range(3))

    @property
    def per_mask(self):
        """kernel_params::per_mask: bit i set when direction i is periodic."""
        return sum(1 << i for i, p in enumerate(self.periodic) if p)

    def __repr__(self):
        return ("MLSettings(relaxation=%r, cycle=%r, nrelax=(%d,%d), num_levels=%d, maxiter=%d, "
                "tol=%g, min_coarse=%d, precision=%r)" % (
                    self.relaxation, self.cycle, self.nrelax_pre, self.nrelax_post, self.num_levels,
                    self.maxiter, self.tol, self.min_coarse, self.precision))
