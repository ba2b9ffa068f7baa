"""Writes tests/golden/oracle_histories.json: residual histories of the CPU
oracle on small seeded cases.  They pin the oracle against drift (the reference
itself cannot be built here: no Fortran compiler or LAPACK) and give the GPU
tests fixed numbers.  Run: python tests/golden/make_fixtures.py"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cedar_b200 import gallery as G  # noqa: E402
from cedar_b200 import problems as P  # noqa: E402

CASES = [
    {"name": "poisson-noise-63-point", "gen": "poisson_noise", "n": 63, "relax": "point",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 12, "tol": 1e-10},
    {"name": "poisson-noise-64-point", "gen": "poisson_noise", "n": 64, "relax": "point",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 12, "tol": 1e-10},
    {"name": "fe-const-63-linexy", "gen": "fe_const", "n": 63, "relax": "line-xy",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 12, "tol": 1e-10},
    {"name": "hetero-63-linexy", "gen": "hetero", "n": 63, "relax": "line-xy",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 8, "tol": 1e-10},
    {"name": "hetero-66-linexy", "gen": "hetero", "n": 66, "relax": "line-xy",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 8, "tol": 1e-10},
    {"name": "hetero-sigma1-65-point", "gen": "hetero_s1", "n": 65, "relax": "point",
     "nrelax_pre": 1, "nrelax_post": 1, "maxiter": 10, "tol": 1e-10},
    {"name": "aniso-5pt-48x40-linex", "gen": "aniso5", "n": 48, "relax": "line-x",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 10, "tol": 1e-10},
    {"name": "aniso-5pt-40x48-liney", "gen": "aniso5y", "n": 48, "relax": "line-y",
     "nrelax_pre": 2, "nrelax_post": 1, "maxiter": 10, "tol": 1e-10},
]


def build_case(case):
    n = case["n"]
    g = case["gen"]
    if g == "poisson_noise":
        so, b = P.poisson_noise(n, seed=0)
    elif g == "fe_const":
        so, b = P.hetero_diffusion(n, sigma=0.0, n_incl=0, aniso=1.0)
    elif g == "hetero":
        so, b = P.hetero_diffusion(n)
    elif g == "hetero_s1":
        so, b = P.hetero_diffusion(n, sigma=1.0, n_incl=0, aniso=1.0)
    elif g == "aniso5":
        so = G.diag_diffusion(n, 40, 1.0, 1e-2)
        b = np.zeros((42, n + 2)); b[1:-1, 1:-1] = np.random.default_rng(4).random((40, n)) * 1e-4
    elif g == "aniso5y":
        so = G.diag_diffusion(40, n, 1e-2, 1.0)
        b = np.zeros((n + 2, 42)); b[1:-1, 1:-1] = np.random.default_rng(4).random((n, 40)) * 1e-4
    else:
        raise ValueError(g)
    kw = {k: case[k] for k in ("relax", "nrelax_pre", "nrelax_post", "maxiter", "tol")}
    return so, b, kw


def main():
    from oracle import oracle as O
    O.build()
    out = {"generator": "tests/golden/make_fixtures.py", "cases": []}
    for case in CASES:
        so, b, kw = build_case(case)
        s = O.Solver(so, **kw)
        x, h = s.solve(b)
        c = dict(case)
        c["history"] = [float(v) for v in h]
        out["cases"].append(c)
        print(case["name"], s.nlevels, " ".join("%.3e" % v for v in h))
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_histories.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
