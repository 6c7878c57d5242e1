"""CPU restatement of the runoff forcing map and the output statistics --
TEST INFRASTRUCTURE.

Only tests/ and bench.py's CPU-baseline leg use this module; the product
(cmfb200.forcing, cmfb200.model statistics) never imports it.

Forcing map.  The reference maps gridded runoff onto catchments with
hydroforge's `build_local_mapping` / `shard_forcing`
(scripts/run_daily_bin.py:98-118).  hydroforge (>= 0.1.0, the pyproject
dependency of the reference) is not in the reference tree, so this restates
the operation from what the reference itself fixes about it: the mapping
table is a CSR matrix [catchments x runoff-grid cells] of areas whose columns
are iy * nx + ix (cmfgpu/params/export_bin.py:955-983, 1071-1075), and the
catchment runoff is that matrix times the grid vector (export_bin.py turns the
same table into CaMa-Flood's inpmat, whose use is the area-weighted sum of
the runoff cells over a catchment, optionally skipping the missing value and
clamping at zero).  Parity pin: `map_grid` is checked against
scipy.sparse.csr_matrix products on the same table.

Every row is summed in entry order in fp64, products and sums rounded
separately, then multiplied by 1 / unit_factor (the reciprocal rounded once)
-- the order the CUDA kernel uses, so fp64 outputs are bit-identical.

Statistics.  `StatsReplay` replays the device statistics (mean over sub-steps
weighted by dt, max, min, last) from per-sub-step snapshots of the state.
"""
from __future__ import annotations

import numpy as np


def map_grid(row_ptr: np.ndarray, col: np.ndarray, weight: np.ndarray, grid: np.ndarray,
             unit_factor: float = 1.0, missing_value=None, clamp_negative: bool = False,
             out_dtype=np.float64) -> np.ndarray:
    """grid [S, G] (any float dtype) -> [S, rows] in out_dtype.

    Vectorised over rows; sequential over the k-th entry of every row, so each
    row's sum runs in entry order."""
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    weight = np.asarray(weight, dtype=np.float64)
    grid = np.asarray(grid)
    S, R = grid.shape[0], row_ptr.size - 1
    lens = np.diff(row_ptr)
    acc = np.zeros((S, R), dtype=np.float64)
    for k in range(int(lens.max()) if R else 0):
        rows = np.flatnonzero(lens > k)
        e = row_ptr[rows] + k
        x = grid[:, col[e]]                      # [S, rows] in the grid dtype
        prod = x.astype(np.float64) * weight[e]  # rounded product
        if missing_value is not None:
            miss = np.isnan(x) | (x == np.asarray(missing_value, dtype=grid.dtype))
            prod = np.where(miss, 0.0, prod)
            acc[:, rows] = np.where(miss, acc[:, rows], acc[:, rows] + prod)
        else:
            acc[:, rows] = acc[:, rows] + prod   # rounded sum
    y = acc * (1.0 / unit_factor)
    if clamp_negative:
        y = np.where(y < 0.0, 0.0, y)
    return y.astype(out_dtype)


def scipy_map(row_ptr, col, weight, grid, num_cols):
    """The same product through scipy.sparse (the pin of map_grid)."""
    from scipy.sparse import csr_matrix
    A = csr_matrix((np.asarray(weight, np.float64), np.asarray(col, np.int64),
                    np.asarray(row_ptr, np.int64)), shape=(len(row_ptr) - 1, num_cols))
    return np.stack([A @ np.asarray(g, np.float64) for g in np.asarray(grid)])


class StatsReplay:
    """Host replay of the device statistics over sub-step snapshots.

    `add(values, dt)` folds the values after one sub-step (dict name -> [N]
    array, fp64) with sub-step length dt; `result(last_values)` returns the
    finished statistics.  Same operation order as the CUDA kernel:
    acc = acc + (x * dt) with separately rounded ops; weight = weight + dt."""

    def __init__(self, spec):
        self.spec = list(spec)                   # [(name, op)]
        self.acc = {}
        self.weight = 0.0

    def add(self, values, dt: float) -> None:
        dt = float(dt)
        self.weight = self.weight + dt
        for name, op in self.spec:
            x = np.asarray(values[name], dtype=np.float64)
            key = (name, op)
            if op == "mean":
                self.acc[key] = self.acc.get(key, np.zeros_like(x)) + x * dt
            elif op == "max":
                a = self.acc.get(key, np.full_like(x, -np.inf))
                self.acc[key] = np.where((x > a) | np.isnan(x), x, a)
            elif op == "min":
                a = self.acc.get(key, np.full_like(x, np.inf))
                self.acc[key] = np.where((x < a) | np.isnan(x), x, a)

    def result(self, last_values) -> dict:
        out = {}
        for name, op in self.spec:
            if op == "mean":
                out[f"{name}_{op}"] = self.acc[(name, op)] / self.weight
            elif op == "last":
                out[f"{name}_{op}"] = np.asarray(last_values[name], dtype=np.float64)
            else:
                out[f"{name}_{op}"] = self.acc[(name, op)]
        return out
