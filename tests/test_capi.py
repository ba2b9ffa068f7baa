"""CPU checks of the C ABI library: it builds, loads, and exports every symbol that
include/cdr_gpu.h declares.  No compute calls (there is no GPU here)."""
import ctypes
import subprocess

import pytest

from cedar_b200 import _lib, build


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    syms = _lib.header_symbols()
    assert "cdr_gpu_residual_2d_f64" in syms
    assert "cdr_gpu_solver_create_2d" in syms
    assert len(syms) >= 30


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in _lib.header_symbols() if s not in exported]
    assert not missing, missing
    for s in _lib.header_symbols():
        assert hasattr(lib, s)


def test_host_only_entry_points(lib):
    s = _lib.Settings()
    assert lib.cdr_gpu_settings_default(ctypes.byref(s)) == 0
    assert (s.relaxation, s.nrelax_pre, s.nrelax_post, s.num_levels, s.maxiter, s.min_coarse) == (0, 2, 1, -1, 10, 3)
    assert s.tol == 1e-8
    assert lib.cdr_gpu_norm_scratch_bytes() > 0
    assert lib.cdr_gpu_version() >= 100


def test_argument_errors_need_no_device(lib):
    # validation runs before any CUDA call
    rc = lib.cdr_gpu_residual_2d_f64(None, 5, None, None, None, 10, 10, 12, None, None, None)
    assert rc == 1  # CDR_ERR_ARG (null pointers)
    rc = lib.cdr_gpu_residual_2d_f64(None, 5, None, None, None, 10, 10, 5, None, None, None)
    assert rc == 2  # CDR_ERR_DIM (pitch < nx+2)
    assert b"pitch" in lib.cdr_gpu_last_error()
    rc = lib.cdr_gpu_restrict_2d_f64(None, None, None, 9, 9, 11, 4, 5, 6, None)
    assert rc == 2  # coarse grid is not the coarsening of the fine grid
    s = _lib.Settings()
    lib.cdr_gpu_settings_default(ctypes.byref(s))
    s.relaxation = 7
    h = ctypes.c_void_p()
    rc = lib.cdr_gpu_solver_create_2d(ctypes.byref(s), ctypes.c_void_p(1), 5, 8, 8, None, ctypes.byref(h))
    assert rc == 1 and b"relaxation" in lib.cdr_gpu_last_error()


def test_config_keys():
    from cedar_b200.config import Config, MLSettings
    ms = MLSettings(Config({"solver": {"relaxation": "line-xy", "cycle": {"nrelax-pre": 3}, "min-coarse": 9,
                                       "tol": 1e-10}}))
    assert ms.relaxation == "line-xy" and ms.nrelax_pre == 3 and ms.nrelax_post == 1
    assert ms.min_coarse == 3  # "min-coarse" is not the key the reference reads
    assert ms.tol == 1e-10 and ms.maxiter == 10
    with pytest.raises(ValueError):
        MLSettings(Config({"solver": {"relaxation": "jacobi"}}))


def test_config_gpu_keys_map_to_settings():
    """The GPU options of the "gpu" object and solver.cycle.type land in
    cdr_gpu_settings; solver.cg-solver is validated but, as in the reference's
    serial solvers, leaves the coarsest-level solve alone."""
    from cedar_b200.config import Config, MLSettings
    from cedar_b200.solver import _settings
    ms = MLSettings(Config({"solver": {"relaxation": "line-xy", "cycle": {"type": "f"}, "cg-solver": "cedar"},
                            "gpu": {"precision": "fp32-ir", "krylov": "fcg", "coarse-solve": "inverse",
                                    "fp32-levels": 2, "fcg-replace": 10, "autotune": False, "line-stream": True,
                                    "line-solve": "sequential"}}))
    s = _settings(ms)
    assert (s.cycle, s.krylov, s.coarse_solve, s.fp32_levels, s.krylov_replace) == (1, 1, 1, 2, 10)
    assert s.precision == _lib.PREC["fp32-ir"]
    assert s.line_flags == _lib.LINES_EXACT | _lib.LINES_NOTUNE | _lib.LINES_STREAM
    s3 = _settings(MLSettings(Config({"solver": {"relaxation": "plane-xyz", "cycle": {"type": "f"}}})), dim=3)
    assert s3.cycle == 1
    with pytest.raises(ValueError):
        MLSettings(Config({"solver": {"cg-solver": "dense"}}))
    with pytest.raises(ValueError):
        MLSettings(Config({"gpu": {"fcg-replace": -1}}))
    # the FP32 cycle's fine-level iterate: FP64 by default, "fp32" turns it off
    assert s.fp64_fine_iterate == 1
    assert _settings(MLSettings(Config({"gpu": {"fine-iterate": "fp32"}}))).fp64_fine_iterate == 0
    with pytest.raises(ValueError):
        MLSettings(Config({"gpu": {"fine-iterate": "fp16"}}))
