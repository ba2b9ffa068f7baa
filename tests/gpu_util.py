"""Helpers for the GPU tests: torch owns device memory, the C ABI computes."""
import ctypes

import numpy as np


def torch():
    import torch as _t
    return _t


def dev(a, dtype=None):
    t = torch()
    a = np.ascontiguousarray(a)
    x = t.from_numpy(a).cuda()
    return x if dtype is None else x.to(dtype)


def ptr(x):
    return ctypes.c_void_p(x.data_ptr()) if x is not None else None


def stream():
    return ctypes.c_void_p(torch().cuda.current_stream().cuda_stream)


def host(x):
    torch().cuda.synchronize()
    return x.double().cpu().numpy()


def padded(a, pitch, dtype=None):
    """Device copy of a Cedar-layout array (..., jj, ii) with rows padded to ``pitch``."""
    t = torch()
    a = np.ascontiguousarray(a)
    shp = a.shape[:-1] + (pitch,)
    out = t.zeros(shp, dtype=t.float64, device="cuda")
    out[..., :a.shape[-1]] = t.from_numpy(a).cuda()
    return out if dtype is None else out.to(dtype)


def rel_err(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b)).max()
    m = np.abs(np.asarray(b)).max()
    return d / m if m > 0 else d
