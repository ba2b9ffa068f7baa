"""Cedar's C interface (include/cedar_capi.h, the calls of the reference's
include/cedar/capi.h) over the GPU solvers.

CPU: every declared function is exported; the handle encoding (kind in the top
four bits) and the error codes of the reference; configs from JSON files;
vertex-based matrix entries land in BoxMG's symmetric storage exactly as the
reference's cedar_mat_set2d puts them (checked through the operator dump).
GPU: a C program written against the interface solves 2D Poisson problems;
its solution equals the oracle's solve of the same operator bit for bit
(sequential line substitutions are not involved: point relaxation), and
cedar_matvec gives the residual.
"""
import ctypes
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from cedar_b200 import _lib
from cedar_b200 import gallery as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cedar_capi.h")

SUCCESS, ERR_TOPO, ERR_KIND, ERR_HANDLE, ERR_MAT, ERR_VEC, ERR_DIM, ERR_STENCIL, ERR_SOLVER, ERR_CONFIG, \
    ERR_FNAME, ERR_CONFIG_PATH = range(12)


class Coord2(ctypes.Structure):
    _fields_ = [("i", ctypes.c_uint), ("j", ctypes.c_uint), ("dir", ctypes.c_int)]


def _cedar():
    from cedar_b200 import build
    build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def _config(tmp_path, tree):
    p = tmp_path / "config.json"
    p.write_text(json.dumps(tree))
    return str(p).encode()


def test_every_declared_function_is_exported():
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    names = sorted(set(re.findall(r"\bint\s+(cedar_[a-z0-9_]+)\s*\(", txt)))
    assert len(names) >= 25
    L = _cedar()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_handles_configs_and_errors(tmp_path):
    L = _cedar()
    I = ctypes.c_int
    conf, topo = I(), I()
    assert L.cedar_config_create(b"/nonexistent/config.json", ctypes.byref(conf)) == ERR_FNAME
    assert conf.value == 0x50000000
    fname = _config(tmp_path, {"solver": {"max-iter": 7, "cycle": {"nrelax-pre": 3}, "relaxation": "line-xy"}})
    assert L.cedar_config_create(fname, ctypes.byref(conf)) == SUCCESS
    assert (conf.value >> 28) == 0x5
    v = I()
    assert L.cedar_config_get_int(conf, b"solver.max-iter", ctypes.byref(v)) == SUCCESS and v.value == 7
    assert L.cedar_config_get_int(conf, b"solver.cycle.nrelax-pre", ctypes.byref(v)) == SUCCESS and v.value == 3
    assert L.cedar_config_get_int(conf, b"solver.nothing", ctypes.byref(v)) == ERR_CONFIG_PATH
    assert L.cedar_log_init(conf) == SUCCESS
    n = 6
    lx = (ctypes.c_uint * 1)(n)
    assert L.cedar_topo_create2d(ctypes.c_long(0), n, n, lx, lx, 2, 1, ctypes.byref(topo)) == ERR_TOPO
    assert L.cedar_topo_create2d(ctypes.c_long(0), n, n, lx, lx, 1, 1, ctypes.byref(topo)) == SUCCESS
    assert (topo.value >> 28) == 0x1
    vec, mat = I(), I()
    assert L.cedar_vec_create2d(conf, ctypes.byref(vec)) == ERR_TOPO  # a config is not a topology
    assert L.cedar_vec_create2d(topo, ctypes.byref(vec)) == SUCCESS and (vec.value >> 28) == 0x4
    ilen, jlen, nd = ctypes.c_uint(), ctypes.c_uint(), I()
    assert L.cedar_vec_len2d(vec, ctypes.byref(ilen), ctypes.byref(jlen)) == SUCCESS
    assert (ilen.value, jlen.value) == (n + 2, n + 2)
    assert L.cedar_vec_getdim(vec, ctypes.byref(nd)) == SUCCESS and nd.value == 2
    assert L.cedar_vec_len3d(vec, ctypes.byref(ilen), ctypes.byref(jlen), ctypes.byref(ilen)) == ERR_DIM
    assert L.cedar_mat_create2d(conf, topo, 1, ctypes.byref(mat)) == SUCCESS and (mat.value >> 28) == 0x3
    t2 = I()
    assert L.cedar_mat_gettopo(mat, ctypes.byref(t2)) == SUCCESS and t2.value == topo.value
    slv = I()
    assert L.cedar_solver_create(vec, ctypes.byref(slv)) == ERR_MAT
    assert slv.value == 0x20000000
    x = I(vec.value)
    assert L.cedar_matvec(mat, conf, x) == ERR_VEC
    assert L.cedar_vec_free(ctypes.byref(x)) == SUCCESS and x.value == 0x40000000
    assert L.cedar_vec_free(ctypes.byref(x)) == ERR_VEC  # the null handle
    assert L.cedar_mat_free(ctypes.byref(mat)) == SUCCESS
    assert L.cedar_topo_free(ctypes.byref(topo)) == SUCCESS
    assert L.cedar_config_free(ctypes.byref(conf)) == SUCCESS


def _set_vertex_stencil(L, mat, A, n, nine):
    """Enter a (n*n x n*n) dense symmetric matrix row by row, vertex-based."""
    dirs = [(0, 0, 0), (1, -1, 0), (2, 0, -1), (8, 1, 0), (6, 0, 1)]
    if nine:
        dirs += [(3, -1, -1), (5, 1, -1), (7, 1, 1), (4, -1, 1)]
    for j in range(n):
        for i in range(n):
            cs, vs = [], []
            for d, di, dj in dirs:
                ii, jj = i + di, j + dj
                if 0 <= ii < n and 0 <= jj < n:
                    cs.append(Coord2(i, j, d))
                    vs.append(A[j * n + i, jj * n + ii])
            arr = (Coord2 * len(cs))(*cs)
            vals = (ctypes.c_double * len(vs))(*vs)
            assert L.cedar_mat_set2d(mat, len(cs), arr, vals) == SUCCESS


@pytest.mark.parametrize("nine", [False, True])
def test_vertex_entries_become_boxmg_storage(tmp_path, nine):
    """A heterogeneous symmetric operator entered vertex by vertex (every row's
    C, W, S, E, N and, nine-point, the four diagonals) gives back Cedar's own
    stored operator: the dump rows equal the gallery operator's rows."""
    L = _cedar()
    I = ctypes.c_int
    n = 7
    rng = np.random.default_rng(4)
    k = np.exp(rng.standard_normal((n + 1, n + 1)))
    so = G.fe_hetero(k, k) if nine else G.diag_diffusion(n, n, 1.3, 0.7)
    A = G.stencil_to_csr(so).toarray()
    conf, topo, mat = I(), I(), I()
    assert L.cedar_config_create(_config(tmp_path, {}), ctypes.byref(conf)) == SUCCESS
    lx = (ctypes.c_uint * 1)(n)
    assert L.cedar_topo_create2d(ctypes.c_long(0), n, n, lx, lx, 1, 1, ctypes.byref(topo)) == SUCCESS
    assert L.cedar_mat_create2d(conf, topo, 1 if nine else 0, ctypes.byref(mat)) == SUCCESS
    _set_vertex_stencil(L, mat, A, n, nine)
    if not nine:  # five-point operators refuse the diagonal directions
        c = (Coord2 * 1)(Coord2(1, 1, 3))
        assert L.cedar_mat_set2d(mat, 1, c, (ctypes.c_double * 1)(1.0)) == ERR_STENCIL
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        assert L.cedar_mat_dump(mat) == SUCCESS
        rows = open("op-0-0.txt").read().splitlines()
    finally:
        os.chdir(cwd)
    assert len(rows) == n * n
    for r, line in enumerate(rows):
        j, i = divmod(r, n)
        vals = [float(v) for v in re.findall(r"-?\d\.\d+e[+-]\d+", line.split(",", 2)[2])]
        # dump order: NW N NE W C E SW S SE (nine-point) / N W C E S (five-point)
        nb = [(-1, 1), (0, 1), (1, 1), (-1, 0), (0, 0), (1, 0), (-1, -1), (0, -1), (1, -1)] if nine else \
            [(0, 1), (-1, 0), (0, 0), (1, 0), (0, -1)]
        for v, (di, dj) in zip(vals, nb):
            ii, jj = i + di, j + dj
            want = A[j * n + i, jj * n + ii] if 0 <= ii < n and 0 <= jj < n else 0.0
            assert abs(v - want) <= 1e-6 * max(1.0, abs(want)), (i, j, di, dj, v, want)
    I2 = I(mat.value)
    assert L.cedar_mat_free(ctypes.byref(I2)) == SUCCESS


@pytest.mark.gpu
@pytest.mark.parametrize("stencil", [5, 9])
def test_c_program_solves_through_the_interface(tmp_path, oracle, stencil):
    """tests/capi/cedar_poisson.c, compiled here and linked to libcdrgpu.so:
    its solve equals the oracle's solve of the same operator bit for bit
    (V(2,1) point relaxation, 10 cycles) and cedar_matvec reports its residual."""
    _cedar()
    exe = tmp_path / "cedar_poisson"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["gcc", "-O2", "-o", str(exe), os.path.join(ROOT, "tests", "capi", "cedar_poisson.c"),
                    "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lcdrgpu", "-Wl,-rpath," + libdir, "-lm"],
                   check=True)
    n = 127
    conf = _config(tmp_path, {"solver": {"relaxation": "point", "max-iter": 10, "tol": 1e-12,
                                         "cycle": {"nrelax-pre": 2, "nrelax-post": 1}}})
    out = tmp_path / "x.bin"
    p = subprocess.run([str(exe), conf.decode(), str(n), str(stencil), str(out)], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    rel = float(p.stdout.split()[-1])
    xb = np.fromfile(str(out), dtype=np.float64).reshape(2, n + 2, n + 2)
    x, b = xb[0], np.ascontiguousarray(xb[1])
    so = G.poisson(n, n) if stencil == 5 else G.fe_hetero(np.ones((n + 1, n + 1)), np.ones((n + 1, n + 1)))
    # the program's operator: 4/-1 (five-point) or 8/-1 (nine-point), unscaled
    if stencil == 5:
        so = np.zeros_like(so); so[0, 1:-1, 1:-1] = 4; so[1, 1:-1, 2:-1] = 1; so[2, 2:-1, 1:-1] = 1
    else:
        so = np.zeros((5, n + 2, n + 2)); so[0, 1:-1, 1:-1] = 8; so[1, 1:-1, 2:-1] = 1; so[2, 2:-1, 1:-1] = 1
        so[3, 2:-1, 2:-1] = 1; so[4, 2:-1, 2:-1] = 1
    # the program's b (its sines round differently from numpy's), checked against the formula
    h = 1.0 / (n + 1)
    idx = np.arange(1, n + 1) * h
    bf = 8 * np.pi ** 2 * np.outer(np.sin(2 * np.pi * idx), np.sin(2 * np.pi * idx)) * h * h
    np.testing.assert_allclose(b[1:-1, 1:-1], bf, rtol=1e-12, atol=1e-18)
    xo, ho = oracle.Solver(so, relax="point", maxiter=10, tol=1e-12).solve(b)
    np.testing.assert_array_equal(x, xo)
    r = oracle.residual(np.ascontiguousarray(so), xo, b)
    # b - A x cancels to ~1e-11 of b: the program's b - matvec(x) and the oracle's fused residual
    # round differently at that level
    assert abs(rel - np.linalg.norm(r) / np.linalg.norm(b)) <= 1e-3 * rel
