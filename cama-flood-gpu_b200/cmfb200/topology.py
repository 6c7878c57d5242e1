"""Topology, masks and derived parameters built at model construction.

Integer/index work here is bit-exact with the reference preprocessing and
module code; the loops run in the native library (libcmfb200 host functions):

* topological order            cmfgpu/params/utils.py:83-138
* upstream CSR                 cmfgpu/params/utils.py:160-206
* initial river depth          cmfgpu/params/utils.py:140-157
* levee base height            cmfgpu/modules/levee.py:140-217
* reservoir masks              cmfgpu/modules/reservoir.py:129-163
* reservoir derived volumes    cmfgpu/modules/reservoir.py:174-206
* dam cold start / path mask   cmfgpu/modules/reservoir.py:208-235

plus the breadth-first catchment order the device kernels need (upstream cells
of every catchment contiguous), its flags and sparse slot tables.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def topological_sort(catchment_id: np.ndarray, downstream_id: np.ndarray) -> np.ndarray:
    cid = np.ascontiguousarray(catchment_id, dtype=np.int64)
    did = np.ascontiguousarray(downstream_id, dtype=np.int64)
    out = np.empty(cid.shape[0], dtype=np.int32)
    rc = _lib.lib().cmf_topo_topological_sort(cid.shape[0], _ptr(cid), _ptr(did), _ptr(out))
    if rc != _lib.CMF_OK:
        raise ValueError("Rings exist and topological sorting is not possible")
    return out


def upstream_csr(downstream_idx: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    n = dn.shape[0]
    indptr = np.empty(n + 1, dtype=np.int32)
    indices = np.empty(max(n, 1), dtype=np.int32)
    _lib.check(_lib.lib().cmf_topo_upstream_csr(n, _ptr(dn), _ptr(indptr), _ptr(indices)),
               "upstream_csr")
    return indptr, indices[: indptr[n]].copy()


def bfs_order(downstream_idx: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(order, up_ptr): order[new] = old index, basin-major breadth-first.

    The upstream cells of new p are [up_ptr[p], upstream_end(p)) where the end
    is up_ptr[p+1], one less when p+1 is a mouth (see upstream_end)."""
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    n = dn.shape[0]
    order = np.empty(n, dtype=np.int32)
    up = np.empty(n + 1, dtype=np.int32)
    rc = _lib.lib().cmf_topo_bfs_order(n, _ptr(dn), _ptr(order), _ptr(up))
    if rc != _lib.CMF_OK:
        raise ValueError("river network has a cycle: some catchment never reaches a mouth")
    return order, up


def init_river_depth(catchment_elevation, river_height, downstream_idx, visit=None) -> np.ndarray:
    ce = np.ascontiguousarray(catchment_elevation, dtype=np.float32)
    rh = np.ascontiguousarray(river_height, dtype=np.float32)
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    out = np.zeros(ce.shape[0], dtype=np.float32)
    vp = None
    if visit is not None:
        visit = np.ascontiguousarray(visit, dtype=np.int32)
        vp = _ptr(visit)
    _lib.check(_lib.lib().cmf_topo_init_river_depth(ce.shape[0], _ptr(ce), _ptr(rh), _ptr(dn),
                                                    vp, _ptr(out)), "init_river_depth")
    return out


def accumulate_upstream(downstream_idx, values) -> np.ndarray:
    """Sum of `values` over each cell and everything upstream of it.  Takes a
    topological order (downstream cells after their upstream cells) or its
    reverse, such as the model's breadth-first order from the mouths."""
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    n = dn.shape[0]
    idx = np.arange(n)
    inner = dn != idx
    if n and inner.any() and (dn[inner] < idx[inner]).all():
        flipped = accumulate_upstream((n - 1 - dn)[::-1], np.asarray(values)[::-1])
        return np.ascontiguousarray(flipped[::-1])
    v = np.ascontiguousarray(values, dtype=np.float64)
    out = np.empty_like(v)
    _lib.check(_lib.lib().cmf_topo_accumulate_upstream(dn.shape[0], _ptr(dn), _ptr(v), _ptr(out)),
               "accumulate_upstream (needs topological order)")
    return out


def accumulate_downstream(downstream_idx, values) -> np.ndarray:
    dn = np.ascontiguousarray(downstream_idx, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.float64)
    out = np.empty_like(v)
    _lib.check(_lib.lib().cmf_topo_accumulate_downstream(dn.shape[0], _ptr(dn), _ptr(v), _ptr(out)),
               "accumulate_downstream (needs topological order)")
    return out


def levee_base_height(flood_depth_table: np.ndarray, levee_catchment_idx: np.ndarray,
                      levee_fraction: np.ndarray) -> np.ndarray:
    """Linear interpolation of the flood-depth table at levee_fraction * K
    (cmfgpu/modules/levee.py:140-217): virtual index 0 is depth 0, index k>0 is
    table[:, k-1]; all arithmetic in float32 as the reference tensors."""
    table = np.asarray(flood_depth_table, dtype=np.float32)
    K = table.shape[-1]
    rows = table[np.asarray(levee_catchment_idx, dtype=np.int64)]
    position = np.asarray(levee_fraction, dtype=np.float32) * np.float32(K)
    position = np.clip(position, np.float32(0.0), np.float32(K)).astype(np.float32)
    lower = np.floor(position).astype(np.int32)
    upper = lower + 1
    frac = (position - lower.astype(np.float32)).astype(np.float32)
    lower_gather = np.maximum(lower - 1, 0)
    lower_val = np.take_along_axis(rows, lower_gather[:, None].astype(np.int64), axis=-1)[:, 0]
    lower_val = np.where(lower == 0, np.float32(0.0), lower_val).astype(np.float32)
    upper_idx = np.minimum(upper - 1, K - 1)
    upper_val = np.take_along_axis(rows, upper_idx[:, None].astype(np.int64), axis=-1)[:, 0]
    return (lower_val + frac * (upper_val - lower_val)).astype(np.float32)


def reservoir_derived(conservation_volume, emergency_volume, normal_outflow,
                      flood_control_outflow) -> dict[str, np.ndarray]:
    """Derived reservoir parameters (cmfgpu/modules/reservoir.py:174-206),
    evaluated with the same float32 torch operations on the host."""
    C = torch.as_tensor(np.asarray(conservation_volume, dtype=np.float32))
    E = torch.as_tensor(np.asarray(emergency_volume, dtype=np.float32))
    Qn = torch.as_tensor(np.asarray(normal_outflow, dtype=np.float32))
    Qf = torch.as_tensor(np.asarray(flood_control_outflow, dtype=np.float32))
    flood_volume = (E - C) / 0.95
    adjustment_volume = C + flood_volume * 0.1
    seconds_per_year = 365.0 * 24 * 60 * 60
    seconds_per_180_days = 180.0 * 24 * 60 * 60
    vyr = Qn * seconds_per_year
    qsto = (C * 0.7 + vyr / 4.0) / seconds_per_180_days
    effective = torch.minimum(Qn, qsto) * 1.5
    adjustment_outflow = (effective + Qf) * 0.5
    return {
        "flood_volume": flood_volume.numpy(),
        "adjustment_volume": adjustment_volume.numpy(),
        "effective_normal_outflow": effective.numpy(),
        "adjustment_outflow": adjustment_outflow.numpy(),
    }


def dam_masks(downstream_idx: np.ndarray, reservoir_catchment_idx: np.ndarray):
    """(is_reservoir, is_dam_related, is_dam_upstream) -- reservoir.py:129-163."""
    dn = np.asarray(downstream_idx, dtype=np.int64)
    n = dn.shape[0]
    is_res = np.zeros(n, dtype=bool)
    is_res[np.asarray(reservoir_catchment_idx, dtype=np.int64)] = True
    downstream_is_dam = is_res[dn]
    not_mouth = dn != np.arange(n)
    upstream = (~is_res) & not_mouth & downstream_is_dam
    related = is_res | upstream
    return is_res, related, related & ~is_res


def bifurcation_incidence(n: int, catchment_idx: np.ndarray, downstream_idx: np.ndarray):
    """Per-catchment list of incident paths: entries 2*path + (cell is the
    downstream end), in path order for each cell."""
    ci = np.asarray(catchment_idx, dtype=np.int64)
    di = np.asarray(downstream_idx, dtype=np.int64)
    P = ci.shape[0]
    cells = np.concatenate([ci, di])
    codes = np.concatenate([2 * np.arange(P), 2 * np.arange(P) + 1]).astype(np.int64)
    order = np.lexsort((codes, cells))
    counts = np.bincount(cells, minlength=n)
    ptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(counts, out=ptr[1:])
    return ptr, codes[order].astype(np.int32)


def upstream_end(up_ptr: np.ndarray, is_mouth: np.ndarray) -> np.ndarray:
    """End of every catchment's upstream range in the bfs_order layout."""
    n = is_mouth.shape[0]
    end = up_ptr[1:].astype(np.int64).copy()
    end[:-1] -= is_mouth[1:].astype(np.int64)
    return end
