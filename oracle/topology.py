"""Network-generation helpers on the CPU oracle -- TEST INFRASTRUCTURE.

The synthetic generator (cmfb200.synthetic.generate) integrates upstream area,
bed elevation and the cold-start river depth with three host helpers.  The
product runs them in libcmfb200; this module runs the oracle's C restatement
of the same loops (oracle/cmf_oracle.c), so that a process that must not load
the product library -- the reference arm of bench.py -- builds the identical
network.  tests/test_oracle_topology.py holds the two bit for bit equal.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import oracle as O


def _fn(name):
    f = getattr(O.lib(), name)
    f.restype = ctypes.c_int
    return f


def _p(a: np.ndarray) -> ctypes.c_void_p:
    # a typed pointer: a bare int would pass as a 32-bit C int and truncate
    # the addresses of large (mmap-allocated) arrays
    return ctypes.c_void_p(a.ctypes.data)


def accumulate_upstream(downstream_idx, values) -> np.ndarray:
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    n = dn.shape[0]
    idx = np.arange(n)
    inner = dn != idx
    if n and inner.any() and (dn[inner] < idx[inner]).all():
        flipped = accumulate_upstream((n - 1 - dn)[::-1], np.asarray(values)[::-1])
        return np.ascontiguousarray(flipped[::-1])
    v = np.ascontiguousarray(values, dtype=np.float64)
    out = np.empty_like(v)
    if _fn("orc_accumulate_upstream")(ctypes.c_int64(n), _p(dn), _p(v), _p(out)):
        raise ValueError("accumulate_upstream needs a topological order")
    return out


def accumulate_downstream(downstream_idx, values) -> np.ndarray:
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.float64)
    out = np.empty_like(v)
    if _fn("orc_accumulate_downstream")(ctypes.c_int64(dn.shape[0]), _p(dn), _p(v), _p(out)):
        raise ValueError("accumulate_downstream needs a topological order")
    return out


def init_river_depth(catchment_elevation, river_height, downstream_idx) -> np.ndarray:
    ce = np.ascontiguousarray(catchment_elevation, dtype=np.float32)
    rh = np.ascontiguousarray(river_height, dtype=np.float32)
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    out = np.zeros(ce.shape[0], dtype=np.float32)
    if _fn("orc_init_river_depth")(ctypes.c_int64(ce.shape[0]), _p(ce), _p(rh), _p(dn), _p(out)):
        raise ValueError("init_river_depth needs a topological order")
    return out
