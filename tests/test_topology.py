"""Topology and index work against golden vectors from the reference's own
code (tests/golden/make_topology_golden.py): bit-exact.  Plus structural
properties of the breadth-first catchment order the kernels rely on."""
from pathlib import Path

import numpy as np
import pytest

from cmfb200 import synthetic as syn, topology

GOLD = np.load(Path(__file__).parent / "golden" / "topology_golden.npz")
CASES = sorted({k.split("_")[0] for k in GOLD.files})


@pytest.mark.parametrize("case", CASES)
def test_topological_sort_matches_reference(case):
    order = topology.topological_sort(GOLD[f"{case}_topo_catchment_id"],
                                      GOLD[f"{case}_topo_downstream_id"])
    np.testing.assert_array_equal(order, GOLD[f"{case}_topo_order"])


@pytest.mark.parametrize("case", CASES)
def test_upstream_csr_matches_reference(case):
    cid = GOLD[f"{case}_topo_catchment_id"]
    did = GOLD[f"{case}_topo_downstream_id"]
    pos = {int(c): i for i, c in enumerate(cid)}
    dn = np.array([pos.get(int(d), i) for i, d in enumerate(did)], dtype=np.int32)
    ptr, ind = topology.upstream_csr(dn)
    np.testing.assert_array_equal(ptr, GOLD[f"{case}_csr_indptr"])
    np.testing.assert_array_equal(ind, GOLD[f"{case}_csr_indices"])


@pytest.mark.parametrize("case", CASES)
def test_init_river_depth_matches_reference(case):
    d = topology.init_river_depth(GOLD[f"{case}_depth_elevation"],
                                  GOLD[f"{case}_depth_river_height"],
                                  GOLD[f"{case}_depth_downstream_idx"])
    np.testing.assert_array_equal(d.view(np.uint32),
                                  GOLD[f"{case}_init_river_depth"].astype(np.float32).view(np.uint32))


@pytest.mark.parametrize("case", CASES)
def test_levee_base_height_matches_reference(case):
    b = topology.levee_base_height(GOLD[f"{case}_levee_table"], GOLD[f"{case}_levee_catchment_idx"],
                                   GOLD[f"{case}_levee_fraction"])
    np.testing.assert_array_equal(b.view(np.uint32),
                                  GOLD[f"{case}_levee_base_height"].view(np.uint32))


@pytest.mark.parametrize("case", CASES)
def test_reservoir_derived_and_masks_match_reference(case):
    der = topology.reservoir_derived(GOLD[f"{case}_res_conservation_volume"],
                                     GOLD[f"{case}_res_emergency_volume"],
                                     GOLD[f"{case}_res_normal_outflow"],
                                     GOLD[f"{case}_res_flood_control_outflow"])
    for k, v in der.items():
        np.testing.assert_array_equal(v.view(np.uint32), GOLD[f"{case}_res_{k}"].view(np.uint32), k)
    masks = topology.dam_masks(GOLD[f"{case}_res_downstream_idx"], GOLD[f"{case}_res_catchment_idx"])
    for name, m in zip(("is_reservoir", "is_dam_related", "is_dam_upstream"), masks):
        np.testing.assert_array_equal(m, GOLD[f"{case}_res_{name}"], name)


def test_topological_sort_rejects_rings():
    with pytest.raises(ValueError):
        topology.topological_sort(np.array([0, 1, 2]), np.array([1, 2, 0]))


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 0), (5000, 4), (20000, 5)])
def test_bfs_order_properties(n, seed):
    net = syn.generate(syn.NetworkSpec(n, seed=seed)) if n > 2 else None
    dn = (net.fields["downstream_id"].astype(np.int32) if net
          else np.arange(n, dtype=np.int32) if n == 1 else np.array([1, 1], np.int32))
    order, up = topology.bfs_order(dn)
    assert np.array_equal(np.sort(order), np.arange(n))
    inv = np.empty(n, dtype=np.int64)
    inv[order] = np.arange(n)
    new_dn = inv[dn[order]]
    mouth = new_dn == np.arange(n)
    end = topology.upstream_end(up, mouth)
    # upstream cells of p are exactly [up[p], end[p])
    for p in range(0, n, max(1, n // 500)):
        kids = np.arange(up[p], end[p])
        assert np.all(new_dn[kids] == p)
        assert np.all(kids != p)
    assert up[-1] == n and np.all(np.diff(up) >= 0)
    assert np.all(up[:-1] > np.arange(n))          # upstream cells follow their parent
    assert np.all(end >= up[:-1])
    assert mouth[0]
    # parents precede children
    assert np.all(new_dn[~mouth] < np.flatnonzero(~mouth))
    # basin-major: every basin occupies one contiguous range starting at its mouth
    root = np.arange(n)
    for p in range(n):
        root[p] = p if mouth[p] else root[new_dn[p]]
    starts = np.flatnonzero(mouth)
    assert np.all(np.diff(root) >= 0)
    assert np.array_equal(np.unique(root), starts)
    # the same CSR as the reference semantics, relabelled
    ptr, ind = topology.upstream_csr(new_dn.astype(np.int32))
    np.testing.assert_array_equal(np.diff(ptr), end - up[:-1])
    np.testing.assert_array_equal(ind, np.flatnonzero(~mouth))


def test_bfs_order_rejects_cycles():
    with pytest.raises(ValueError):
        topology.bfs_order(np.array([1, 2, 0, 3], dtype=np.int32))


def test_bifurcation_incidence():
    ci = np.array([0, 2, 0, 4])
    di = np.array([3, 0, 4, 1])
    ptr, codes = topology.bifurcation_incidence(6, ci, di)
    per_cell = {c: sorted(codes[ptr[c]:ptr[c + 1]].tolist()) for c in range(6)}
    assert per_cell[0] == [0, 3, 4]
    assert per_cell[1] == [7]
    assert per_cell[2] == [2]
    assert per_cell[3] == [1]
    assert per_cell[4] == [5, 6]
    assert per_cell[5] == []
