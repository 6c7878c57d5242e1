"""Generate tests/golden/forcing_small.npz: a runoff mapping table, a chunk of
gridded runoff and the catchment runoff it maps to.

    python tests/golden/make_forcing_golden.py

hydroforge (the reference's forcing layer) is not part of the reference tree,
so the expected values come from two computations independent of the code
under test: scipy.sparse CSR products for the plain and unit-converted maps,
and explicit Python loops over the table for the missing-value / clamp rules
(entries whose runoff is NaN or the missing value are left out; the sum is
scaled by 1 / unit_factor, the reciprocal rounded once; negative sums become
zero).  The table uses the reference's `.npz` keys
(cmfgpu/params/export_bin.py:955-983).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "cama-flood-gpu_b200"))

from cmfb200 import synthetic as syn  # noqa: E402

MISSING = np.float32(-9999.0)
UNIT = 86400000.0
GRID = (12, 20)


def build():
    net = syn.generate(syn.NetworkSpec(300, seed=77))
    table = syn.runoff_mapping(net, GRID, seed=5, extra_rows=25)
    rng = np.random.default_rng(2024)
    grid = syn.gridded_runoff(GRID, 3, seed=11).reshape(3, -1)
    # signed values, NaN and the missing value on a few cells
    grid[:, rng.choice(grid.shape[1], 12, replace=False)] *= -1.0
    grid[:, rng.choice(grid.shape[1], 6, replace=False)] = np.nan
    grid[:, rng.choice(grid.shape[1], 6, replace=False)] = MISSING
    clean = np.where(np.isnan(grid) | (grid == MISSING), 0.0, grid).astype(np.float32)

    n_rows, G = (int(x) for x in table["matrix_shape"])
    A = csr_matrix((table["sparse_data"], table["sparse_indices"], table["sparse_indptr"]),
                   shape=(n_rows, G))
    plain = np.stack([A @ g.astype(np.float64) for g in clean])
    unit = plain * (1.0 / UNIT)

    # missing / clamp rules by explicit loops (on the raw grid)
    ptr, idx, w = table["sparse_indptr"], table["sparse_indices"], table["sparse_data"]
    rule = np.zeros((grid.shape[0], n_rows))
    for s in range(grid.shape[0]):
        for r in range(n_rows):
            acc = 0.0
            for e in range(ptr[r], ptr[r + 1]):
                x = grid[s, idx[e]]
                if np.isnan(x) or x == MISSING:
                    continue
                acc = acc + float(x) * float(w[e])
            acc = acc * (1.0 / UNIT)
            rule[s, r] = 0.0 if acc < 0.0 else acc
    return dict(table, grid_clean=clean, grid_raw=grid, expected_plain=plain,
                expected_unit=unit, expected_rules=rule, missing_value=np.float32(MISSING),
                unit_factor=np.float64(UNIT), grid_shape=np.array(GRID))


if __name__ == "__main__":
    out = Path(__file__).resolve().parent / "forcing_small.npz"
    np.savez_compressed(out, **build())
    print("wrote", out)
