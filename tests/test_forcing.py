"""Runoff forcing map, host side (no GPU): the oracle against the golden
fixture and scipy, the mapping-table reader (row selection in model order,
missing catchments, malformed tables) and the statistics replay rules."""
from pathlib import Path

import numpy as np
import pytest

from cmfb200 import synthetic as syn
from cmfb200.forcing import load_mapping_table, local_csr
from oracle import forcing as OF

GOLDEN = Path(__file__).resolve().parent / "golden" / "forcing_small.npz"


def _golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def _table_rows(g):
    """(row_ptr, col, weight) of the whole table in table order."""
    return g["sparse_indptr"], g["sparse_indices"], g["sparse_data"]


def test_oracle_matches_golden_plain_and_unit():
    g = _golden()
    rp, col, w = _table_rows(g)
    np.testing.assert_array_equal(OF.map_grid(rp, col, w, g["grid_clean"]), g["expected_plain"])
    np.testing.assert_array_equal(OF.map_grid(rp, col, w, g["grid_clean"], unit_factor=float(g["unit_factor"])),
                                  g["expected_unit"])


def test_oracle_matches_golden_missing_and_clamp():
    g = _golden()
    rp, col, w = _table_rows(g)
    got = OF.map_grid(rp, col, w, g["grid_raw"], unit_factor=float(g["unit_factor"]),
                      missing_value=g["missing_value"], clamp_negative=True)
    np.testing.assert_array_equal(got, g["expected_rules"])


def test_oracle_equals_scipy_on_random_tables():
    for seed in range(3):
        net = syn.generate(syn.NetworkSpec(2000, seed=seed))
        tab = syn.runoff_mapping(net, (30, 50), seed=seed, max_cells=4)
        rp, col, w, G = local_csr(tab, net.fields["catchment_id"])
        grid = syn.gridded_runoff((30, 50), 4, seed=seed).reshape(4, -1).astype(np.float64)
        np.testing.assert_array_equal(OF.map_grid(rp, col, w, grid), OF.scipy_map(rp, col, w, grid, G))


def test_local_rows_follow_desired_order():
    g = _golden()
    ids = g["catchment_ids"]
    rng = np.random.default_rng(0)
    want = rng.permutation(ids)[: ids.size // 2]
    rp, col, w, G = local_csr(g, want)
    assert G == int(g["matrix_shape"][1])
    # row r of the local table is the table row of want[r], entries in table order
    for r, cid in enumerate(want):
        src = int(np.flatnonzero(ids == cid)[0])
        a, b = g["sparse_indptr"][src], g["sparse_indptr"][src + 1]
        np.testing.assert_array_equal(col[rp[r]:rp[r + 1]], g["sparse_indices"][a:b])
        np.testing.assert_array_equal(w[rp[r]:rp[r + 1]], g["sparse_data"][a:b])
    assert col.dtype == np.int32 and w.dtype == np.float64 and rp.dtype == np.int64


def test_missing_catchment_raises_or_maps_to_empty_row():
    g = _golden()
    want = np.concatenate([g["catchment_ids"][:5], [10 ** 9]])
    with pytest.raises(ValueError, match="not in the runoff mapping table"):
        local_csr(g, want)
    rp, col, w, _ = local_csr(g, want, allow_missing=True)
    assert rp[-1] == rp[-2]                  # last row empty


def test_empty_desired_set():
    g = _golden()
    rp, col, w, _ = local_csr(g, np.zeros(0, dtype=np.int64))
    assert rp.tolist() == [0] and col.size == 0 and w.size == 0


@pytest.mark.parametrize("break_it", ["dup_ids", "bad_col", "bad_ptr", "bad_shape", "missing_key"])
def test_malformed_tables_are_rejected(break_it):
    g = _golden()
    t = dict(g)
    if break_it == "dup_ids":
        t["catchment_ids"] = t["catchment_ids"].copy()
        t["catchment_ids"][1] = t["catchment_ids"][0]
    elif break_it == "bad_col":
        t["sparse_indices"] = t["sparse_indices"].copy()
        t["sparse_indices"][3] = int(t["matrix_shape"][1])
    elif break_it == "bad_ptr":
        t["sparse_indptr"] = t["sparse_indptr"].copy()
        t["sparse_indptr"][-1] += 1
    elif break_it == "bad_shape":
        t["coord_lon"] = np.zeros(t["coord_lon"].size + 1)
    elif break_it == "missing_key":
        del t["sparse_data"]
    with pytest.raises(ValueError):
        local_csr(load_mapping_table(t), t["catchment_ids"][:3] if "catchment_ids" in t else [])


def test_mapping_table_roundtrips_through_npz(tmp_path):
    net = syn.generate(syn.NetworkSpec(500, seed=4))
    tab = syn.runoff_mapping(net, (10, 16), seed=4, extra_rows=7)
    p = tmp_path / "runoff_mapping_bin.npz"
    np.savez(p, **tab)
    a = local_csr(load_mapping_table(p), net.fields["catchment_id"])
    b = local_csr(tab, net.fields["catchment_id"])
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    # every model catchment gets its whole area (weights split the area)
    rp, col, w, _ = a
    area = np.add.reduceat(w, rp[:-1]) if w.size else np.zeros(0)
    np.testing.assert_allclose(area, net.fields["catchment_area"].astype(np.float64), rtol=1e-12)


def test_column_convention_matches_inpmat_indices():
    """Columns are iy * nx + ix (cmfgpu/params/export_bin.py:1071-1075)."""
    g = _golden()
    ny, nx = (int(x) for x in g["grid_shape"])
    col = g["sparse_indices"]
    ix, iy = col % nx, col // nx
    assert ix.max() < nx and iy.max() < ny
    assert g["coord_lon"].size == nx and g["coord_lat"].size == ny


def test_stats_replay_rules():
    r = OF.StatsReplay([("v", "mean"), ("v", "max"), ("v", "min"), ("v", "last")])
    r.add({"v": np.array([1.0, np.nan])}, 2.0)
    r.add({"v": np.array([3.0, 1.0])}, 1.0)
    out = r.result({"v": np.array([3.0, 1.0])})
    assert out["v_mean"][0] == (1.0 * 2.0 + 3.0 * 1.0) / 3.0
    assert np.isnan(out["v_mean"][1]) and np.isnan(out["v_max"][1]) and np.isnan(out["v_min"][1])
    assert out["v_max"][0] == 3.0 and out["v_min"][0] == 1.0 and out["v_last"][0] == 3.0
