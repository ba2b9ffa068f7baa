"""ctypes binding of ``libcdrgpu.so`` (the C ABI declared in include/cdr_gpu.h).

The library is built in-tree by :mod:`cedar_b200.build`.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcdrgpu.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "cdr_gpu.h")

CDR_OK = 0
DOWN, UP = 0, 1
RELAX = {"point": 0, "line-x": 1, "line-y": 2, "line-xy": 3,
         "plane-xy": 4, "plane-xz": 5, "plane-yz": 6, "plane-xyz": 7}
PREC = {"fp64": 0, "fp32-ir": 1}
KRYLOV = {"none": 0, "fcg": 1}
COARSE = {"banded": 0, "inverse": 1}
DIR_X, DIR_Y = 0, 1
LINES_EXACT = 1
LINES_NOTUNE = 2
LINES_STREAM = 4
LINES_ZERO_START = 8
LINES_YPAIR = 16
LINES_YPACKED = 32

_lib = None


class CdrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cdr_gpu error %d: %s" % (code, msg))
        self.code = code


class Settings(ctypes.Structure):
    """``cdr_gpu_settings`` (mirrors ml_settings, include/cedar/multilevel_settings.h:28-50)."""
    _fields_ = [("relaxation", ctypes.c_int), ("nrelax_pre", ctypes.c_int),
                ("nrelax_post", ctypes.c_int), ("num_levels", ctypes.c_int),
                ("maxiter", ctypes.c_int), ("tol", ctypes.c_double),
                ("min_coarse", ctypes.c_int), ("precision", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("line_flags", ctypes.c_int), ("fuse_coarse", ctypes.c_int),
                ("krylov", ctypes.c_int), ("coarse_solve", ctypes.c_int), ("fp32_levels", ctypes.c_int),
                ("cycle", ctypes.c_int), ("krylov_replace", ctypes.c_int), ("periodic", ctypes.c_int),
                ("fp64_fine_iterate", ctypes.c_int)]


def header_symbols():
    """Names of every entry point declared in include/cdr_gpu.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cdr_gpu_[a-z0-9_]+)\s*\(", txt)))


def load(path=LIB_PATH):
    """Load the library (no build).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("cedar_b200: %s is missing; run `python -m cedar_b200.build` "
                           "(there is no CPU fallback)" % path)
    L = ctypes.CDLL(path)
    P, I, D, Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    S = ctypes.c_void_p  # cudaStream_t
    sig = {
        "cdr_gpu_last_error": (ctypes.c_char_p, []),
        "cdr_gpu_version": (I, []),
        "cdr_gpu_launch_count": (ctypes.c_longlong, []),
        "cdr_gpu_lines_shape": (I, [I, I, I, I, I, I, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "cdr_gpu_lines_set_shape": (I, [I, I, I, I, I, I, I, I]),
        "cdr_gpu_lines_stream_status": (I, [S]),
        "cdr_gpu_set_wait_limit_ns": (I, [ctypes.c_longlong]),
        "cdr_gpu_inject_timeouts": (I, [ctypes.c_uint, ctypes.c_uint]),
        "cdr_gpu_norm_scratch_bytes": (Z, []),
        "cdr_gpu_lines_sync_words": (Z, [I]),
        "cdr_gpu_settings_default": (I, [ctypes.POINTER(Settings)]),
        "cdr_gpu_solver_create_2d": (I, [ctypes.POINTER(Settings), P, I, I, I, S, ctypes.POINTER(P)]),
        "cdr_gpu_solver_destroy": (I, [P]),
        "cdr_gpu_solver_create_2d_device": (I, [ctypes.POINTER(Settings), P, I, I, I, I, S, ctypes.POINTER(P)]),
        "cdr_gpu_solver_resetup_device": (I, [P, P, I]),
        "cdr_gpu_fe_assemble_2d_f64": (I, [P, P, I, P, I, I, I, S]),
        "cdr_gpu_fe_grad_2d_f64": (I, [P, P, I, I, I, P, P, I, S]),
        "cdr_gpu_fe_assemble_3d_f64": (I, [P, I, I, P, I, I, I, I, S]),
        "cdr_gpu_solver_solve": (I, [P, P, P, ctypes.POINTER(I), P, I]),
        "cdr_gpu_solver_solve_device": (I, [P, P, P, I, ctypes.POINTER(I), P, I]),
        "cdr_gpu_solver_vcycle_device": (I, [P, P, P, I]),
        "cdr_gpu_solver_nlevels": (I, [P]),
        "cdr_gpu_solver_level": (I, [P, I, I, ctypes.POINTER(P)] + [ctypes.POINTER(I)] * 5),
        "cdr_gpu_solver_timings": (I, [P, ctypes.POINTER(D), ctypes.POINTER(D)]),
        "cdr_gpu_solver_level_get": (I, [P, I, I, P, Z]),
    }
    for suf in ("f64", "f32"):
        sig.update({
            "cdr_gpu_residual_2d_" + suf: (I, [P, I, P, P, P, I, I, I, P, P, S]),
            "cdr_gpu_setup_recip_2d_" + suf: (I, [P, P, I, I, I, S]),
            "cdr_gpu_relax_point_2d_" + suf: (I, [P, I, P, P, P, I, I, I, I, S]),
            "cdr_gpu_setup_lines_2d_" + suf: (I, [P, I, P, I, I, I, I, I, P, S]),
            "cdr_gpu_relax_lines_2d_" + suf: (I, [P, I, P, P, P, I, I, I, I, I, I, I, S]),
            "cdr_gpu_relax_lines_2d_sync_" + suf: (I, [P, I, P, P, P, I, I, I, I, I, I, I, P, S]),
            "cdr_gpu_pack_ylines_2d_" + suf: (I, [P, I, P, I, I, I, I, S]),
            "cdr_gpu_restrict_2d_" + suf: (I, [P, P, P, I, I, I, I, I, I, S]),
            "cdr_gpu_interp_add_2d_" + suf: (I, [P, P, P, P, P, I, I, I, I, I, I, S]),
            "cdr_gpu_solve_cg_2d_" + suf: (I, [P, P, P, I, I, I, S]),
        })
    sig.update({
        "cdr_gpu_residual_2d_f64_noalloc": (I, [P, I, P, P, P, I, I, I, P, S]),
        "cdr_gpu_setup_interp_2d_f64": (I, [P, I, P, I, I, I, I, I, I, S]),
        "cdr_gpu_galerkin_2d_f64": (I, [P, I, P, P, I, I, I, I, I, I, S]),
        "cdr_gpu_setup_cg_2d_f64": (I, [P, I, I, I, I, P, P, S]),
        # 3D
        "cdr_gpu_residual_3d_f64": (I, [P, I, P, P, P, I, I, I, I, P, P, S]),
        "cdr_gpu_residual_3d_f32": (I, [P, I, P, P, P, I, I, I, I, P, P, S]),
        "cdr_gpu_setup_recip_3d_f64": (I, [P, P, I, I, I, I, S]),
        "cdr_gpu_relax_point_3d_f64": (I, [P, I, P, P, P, I, I, I, I, I, S]),
        "cdr_gpu_relax_point_3d_f32": (I, [P, I, P, P, P, I, I, I, I, I, S]),
        "cdr_gpu_restrict_3d_f64": (I, [P, P, P] + [I] * 8 + [S]),
        "cdr_gpu_interp_add_3d_f64": (I, [P, P, P, P, P] + [I] * 8 + [S]),
        "cdr_gpu_setup_interp_3d_f64": (I, [P, I, P] + [I] * 8 + [S]),
        "cdr_gpu_galerkin_3d_f64": (I, [P, I, P, P] + [I] * 8 + [S]),
        "cdr_gpu_setup_cg_3d_f64": (I, [P, I, I, I, I, I, P, P, S]),
        "cdr_gpu_solve_cg_3d_f64": (I, [P, P, P, I, I, I, I, S]),
        "cdr_gpu_solver3_create": (I, [ctypes.POINTER(Settings), P, I, I, I, I, S, ctypes.POINTER(P)]),
        "cdr_gpu_solver3_create_device": (I, [ctypes.POINTER(Settings), P, I, I, I, I, I, S, ctypes.POINTER(P)]),
        "cdr_gpu_solver3_destroy": (I, [P]),
        "cdr_gpu_solver3_solve": (I, [P, P, P, ctypes.POINTER(I), P, I]),
        "cdr_gpu_solver3_solve_device": (I, [P, P, P, I, ctypes.POINTER(I), P, I]),
        "cdr_gpu_solver3_nlevels": (I, [P]),
        "cdr_gpu_solver3_level": (I, [P, I, I, ctypes.POINTER(P)] + [ctypes.POINTER(I)] * 4),
        "cdr_gpu_solver3_level_get": (I, [P, I, I, P, Z]),
        "cdr_gpu_solver3_timings": (I, [P, ctypes.POINTER(D), ctypes.POINTER(D)]),
        # batches of 2D problems
        "cdr_gpu_batch2d_create": (I, [ctypes.POINTER(Settings), P, I, I, I, I, I, S, ctypes.POINTER(P)]),
        "cdr_gpu_batch2d_destroy": (I, [P]),
        "cdr_gpu_batch2d_solve_device": (I, [P, P, P, I, P, P, P]),
        "cdr_gpu_batch2d_nlevels": (I, [P]),
        "cdr_gpu_batch2d_timings": (I, [P, ctypes.POINTER(D), ctypes.POINTER(D)]),
        "cdr_gpu_batch2d_resetup_device": (I, [P, P, I]),
        # independent problems of several sizes
        "cdr_gpu_batchmix_create": (I, [ctypes.POINTER(Settings), I, P, P, P, P, P, P, S, ctypes.POINTER(P)]),
        "cdr_gpu_batchmix_destroy": (I, [P]),
        "cdr_gpu_batchmix_solve_device": (I, [P, P, P, P, P, P, P]),
        "cdr_gpu_batchmix_timings": (I, [P, ctypes.POINTER(D), ctypes.POINTER(D)]),
        "cdr_gpu_batchmix_sizes": (I, [P]),
        "cdr_gpu_batchmix_cycle_launches": (ctypes.c_longlong, [P]),
    })
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != CDR_OK:
        msg = load().cdr_gpu_last_error()
        raise CdrError(rc, msg.decode() if msg else "")
    return rc
