"""Independent problems of several grid sizes solved together (cdr_gpu_batchmix_*).

Each problem must end where its own single-size batch (cdr_gpu_batch2d_*) ends:
the same iterate bit for bit, the same number of cycles and the same final
relative residual, whatever other sizes share the launches.  Sizes whose
hierarchies merge at different levels (odd and even edges) and classes of one
problem are covered.  The mixed batch reports the launches of its captured
cycle.
"""
import numpy as np
import pytest

from cedar_b200.config import Config
from tests.gpu_util import host
from tests.test_gpu_batch import _batch, _device

pytestmark = pytest.mark.gpu


def _conf(relax="line-xy", tol=1e-8, fuse=32):
    return Config({"solver": {"relaxation": relax, "max-iter": 40, "tol": tol,
                              "cycle": {"nrelax-pre": 1, "nrelax-post": 1}},
                   "gpu": {"precision": "fp32-ir", "fuse-coarse": fuse}})


# The classes of the second case fuse their coarse levels from different sizes
# (16 for the 31 class, 32 for the others), so the mixed batch runs every level
# with separate launches: it is compared with single-size batches that do the
# same (gpu.fuse-coarse = 0).
@pytest.mark.parametrize("sizes,relax,fuse", [([(127, 3), (63, 5), (255, 2)], "line-xy", 32),
                                              ([(64, 2), (127, 1), (31, 4)], "line-xy", 0),
                                              ([(95, 3), (47, 2)], "point", 32)])
def test_mixed_batch_equals_single_size_batches(sizes, relax, fuse):
    import torch
    from cedar_b200.solver import BatchSolver2D, MixedBatchSolver2D
    conf = _conf(relax, fuse=fuse)
    classes, data = [], []
    for k, (n, nb) in enumerate(sizes):
        ops, rhs = _batch(n, n, nb, 5, seed=200 + 10 * k)
        pitch = ((n + 2 + 7) // 8) * 8
        so, b = _device(ops, pitch), _device(rhs, pitch)
        data.append((so, b, pitch, n, nb))
        classes.append((so.data_ptr(), 5, n, n, pitch, nb))
    mb = MixedBatchSolver2D(classes, conf)
    xs = [b.clone().zero_() for (_, b, _, _, _) in data]
    mb.solve_device([d[1].data_ptr() for d in data], [x.data_ptr() for x in xs])
    assert mb.cycle_launches > 0
    assert mb.nsizes >= len(sizes)
    first = 0
    for (so, b, pitch, n, nb), x in zip(data, xs):
        s = BatchSolver2D(so.data_ptr(), 5, n, n, pitch, nb, conf)
        xr = b.clone().zero_()
        s.solve_device(b.data_ptr(), xr.data_ptr())
        np.testing.assert_array_equal(host(x), host(xr))
        np.testing.assert_array_equal(mb.iters[first:first + nb], s.iters)
        np.testing.assert_array_equal(mb.rel[first:first + nb], s.rel)
        assert np.all(s.rel < 1e-8)
        first += nb
        s.close()
    assert np.all(mb.done_ms > 0)
    mb.close()


def test_mixed_batch_rejects_fp64_and_bad_classes():
    import torch
    from cedar_b200 import _lib
    from cedar_b200.solver import MixedBatchSolver2D
    ops, rhs = _batch(31, 31, 2, 5, seed=5)
    so = _device(ops, 40)
    with pytest.raises(_lib.CdrError):
        MixedBatchSolver2D([(so.data_ptr(), 5, 31, 31, 40, 2)],
                           Config({"solver": {"relaxation": "line-xy"}, "gpu": {"precision": "fp64"}}))
    with pytest.raises(_lib.CdrError):
        MixedBatchSolver2D([(so.data_ptr(), 5, 31, 31, 20, 2)], _conf())
