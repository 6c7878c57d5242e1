"""Runoff forcing map on the GPU (cmf_forcing_apply through cmfb200.forcing)
against the oracle (oracle/forcing.py) and the golden fixture: bit-exact in
fp64, and fp32 outputs equal to the fp64 result rounded once.  At the size of
the 6M-catchment workload: linearity and the volume identity
sum_r out[r] = sum_c grid[c] * (sum of the weights on column c)."""
from pathlib import Path

import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn
from cmfb200.forcing import (MappedForcing, RunoffMapping, apply_mapping, build_local_mapping,
                             local_csr, shard_forcing)
from oracle import forcing as OF

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "forcing_small.npz"


def _golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def _whole_table(g, device):
    """The golden table with rows in table order (desired = its own ids)."""
    return build_local_mapping(g, g["catchment_ids"], device)


def test_golden_plain_unit_and_rules(device):
    g = _golden()
    m = _whole_table(g, device)
    clean = torch.as_tensor(g["grid_clean"], device=device)
    raw = torch.as_tensor(g["grid_raw"], device=device)
    got = apply_mapping(m, clean.double(), dtype=torch.float64)
    np.testing.assert_array_equal(got.cpu().numpy(), g["expected_plain"])
    got = apply_mapping(m, clean, dtype=torch.float64, unit_factor=float(g["unit_factor"]))
    np.testing.assert_array_equal(got.cpu().numpy(), g["expected_unit"])
    got = apply_mapping(m, raw, dtype=torch.float64, unit_factor=float(g["unit_factor"]),
                        missing_value=float(g["missing_value"]), clamp_negative=True)
    np.testing.assert_array_equal(got.cpu().numpy(), g["expected_rules"])
    # [T, ny, nx] input gives the same as [T, ny*nx]
    ny, nx = (int(x) for x in g["grid_shape"])
    got2 = apply_mapping(m, raw.reshape(-1, ny, nx), dtype=torch.float64,
                         unit_factor=float(g["unit_factor"]), missing_value=float(g["missing_value"]),
                         clamp_negative=True)
    assert torch.equal(got, got2)


@pytest.mark.parametrize("grid_dtype", [np.float32, np.float64])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("steps", [1, 5, 8])
def test_model_order_matches_oracle(grid_dtype, out_dtype, steps, device):
    net = syn.generate(syn.NetworkSpec(20_000, seed=8, bifurcation_paths=100))
    model = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules)
    tab = syn.runoff_mapping(net, (60, 90), seed=3, extra_rows=500)
    cid = model.base.catchment_id.cpu().numpy()
    m = build_local_mapping(tab, cid, device)
    grid = syn.gridded_runoff((60, 90), steps, seed=steps).astype(grid_dtype)
    got = apply_mapping(m, torch.as_tensor(grid, device=device), dtype=out_dtype, unit_factor=86400000.0)
    rp, col, w, _ = local_csr(tab, cid)
    ref = OF.map_grid(rp, col, w, grid.reshape(steps, -1), unit_factor=86400000.0,
                      out_dtype=np.float64 if out_dtype == torch.float64 else np.float32)
    np.testing.assert_array_equal(got.cpu().numpy(), ref)


@pytest.mark.parametrize("members", [1, 3, 4])
def test_members_layout(members, device):
    net = syn.generate(syn.NetworkSpec(5_000, seed=12))
    tab = syn.runoff_mapping(net, (30, 40), seed=12)
    cid = net.fields["catchment_id"][::-1].copy()
    m = build_local_mapping(tab, cid, device)
    grid = syn.gridded_runoff((30, 40), 3, seed=1, members=members)    # [T, M, ny, nx]
    got = apply_mapping(m, torch.as_tensor(grid, device=device), dtype=torch.float64)
    assert tuple(got.shape) == (3, cid.size, members)
    rp, col, w, _ = local_csr(tab, cid)
    for mm in range(members):
        ref = OF.map_grid(rp, col, w, grid[:, mm].reshape(3, -1))
        np.testing.assert_array_equal(got[:, :, mm].cpu().numpy(), ref)


def test_empty_rows_and_out_of_range_columns_flag_status(device):
    g = _golden()
    want = np.concatenate([g["catchment_ids"][:10], [10 ** 9]])
    m = build_local_mapping(g, want, device, allow_missing=True)
    clean = torch.as_tensor(g["grid_clean"], device=device)
    out = apply_mapping(m, clean, dtype=torch.float64)
    assert torch.all(out[:, -1] == 0)
    # a column outside the grid (built here on purpose; the reader rejects
    # such tables) is skipped by the kernel's bounds check and reported
    bad_col = m.col.clone()
    bad_col[0] = m.num_cols + 5
    bad = RunoffMapping(m.row_ptr, bad_col, m.weight, m.num_cols)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    out_bad = apply_mapping(bad, clean, dtype=torch.float64, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) & 4
    rp, col, w, _ = local_csr(g, want, allow_missing=True)
    keep = np.ones(col.size, bool)
    keep[0] = False
    ref = OF.map_grid(rp, np.where(keep, col, 0), np.where(keep, w, 0.0), g["grid_clean"])
    # entry 0 dropped: same as a zero weight on a valid column up to the
    # sign of zero; compare values
    np.testing.assert_array_equal(out_bad.cpu().numpy() + 0.0, ref + 0.0)


def test_zero_steps_and_errors(device):
    g = _golden()
    m = _whole_table(g, device)
    out = apply_mapping(m, torch.zeros((0, m.num_cols), device=device), dtype=torch.float32)
    assert out.shape == (0, m.num_rows)
    with pytest.raises(ValueError):
        apply_mapping(m, torch.zeros((2, m.num_cols + 1), device=device))
    with pytest.raises(ValueError):
        apply_mapping(m, torch.zeros((2, m.num_cols)))               # host tensor
    from cmfb200._lib import CmfError
    with pytest.raises(CmfError):
        apply_mapping(m, torch.zeros((2, m.num_cols), device=device), unit_factor=0.0)


def test_shard_forcing_drives_the_model_like_host_mapped_runoff(device):
    """scripts/run_daily_bin.py:114-124 with the device map: identical states
    to a run fed the oracle-mapped runoff."""
    net = syn.generate(syn.NetworkSpec(8_000, seed=31, bifurcation_paths=60, levee_fraction=0.2,
                                       reservoirs=6))
    kw = dict(device=device, input_proxy=net.fields, opened_modules=net.opened_modules)
    a, b = CaMaFlood(**kw), CaMaFlood(**kw)

    class Dataset(MappedForcing):
        unit_factor = 86400000.0

    ds = Dataset()
    tab = syn.runoff_mapping(net, (40, 60), seed=31)
    local = ds.build_local_mapping(tab, a.base.catchment_id.cpu().numpy(), device)
    chunk = syn.gridded_runoff((40, 60), 3, seed=9)
    mapped = ds.shard_forcing(torch.as_tensor(chunk).to(device), local, dtype=a.base.runoff.dtype)
    rp, col, w, _ = local_csr(tab, a.base.catchment_id.cpu().numpy())
    host = OF.map_grid(rp, col, w, chunk.reshape(3, -1), unit_factor=86400000.0, out_dtype=np.float32)
    for t in range(3):
        a.set_inputs(mapped[t])
        a.step_advance()
        b.set_inputs(torch.as_tensor(host[t]).to(device))
        b.step_advance()
    torch.cuda.synchronize()
    sa, sb = a.state_tensors(), b.state_tensors()
    for k in sa:
        assert torch.equal(sa[k], sb[k]), k


def test_full_size_linearity_and_volume(device):
    """6M catchments on a 0.25-degree grid: properties that need no oracle."""
    net = syn.generate(syn.NetworkSpec(6_000_000, seed=2))
    grid_shape = (720, 1440)
    tab = syn.runoff_mapping(net, grid_shape, seed=2)
    m = build_local_mapping(tab, net.fields["catchment_id"], device)
    x = torch.as_tensor(syn.gridded_runoff(grid_shape, 2, seed=4), device=device).double()
    y = shard_forcing(x, m, dtype=torch.float64)
    # volume: sum over catchments == grid dotted with the column weight sums
    colsum = torch.zeros(m.num_cols, dtype=torch.float64, device=device)
    colsum.index_add_(0, m.col.long(), m.weight)
    vol = x.reshape(2, -1) @ colsum
    torch.testing.assert_close(y.sum(dim=1), vol, rtol=1e-12, atol=0)
    # linearity: map(2x + x') == 2 map(x) + map(x')
    y2 = shard_forcing(2.0 * x[:1] + x[1:], m, dtype=torch.float64)
    torch.testing.assert_close(y2[0], 2.0 * y[0] + y[1], rtol=1e-13, atol=1e-9)
    # a spot check of rows against the oracle
    rp, col, w, _ = local_csr(tab, net.fields["catchment_id"][:2000])
    ref = OF.map_grid(rp, col, w, x.reshape(2, -1).cpu().numpy())
    np.testing.assert_array_equal(y[:, :2000].cpu().numpy(), ref)


@pytest.mark.parametrize("grid_dtype", [np.float32, np.float64])
def test_rows_with_many_entries(grid_dtype, device):
    """Rows of up to 9 entries (a 3x3 block of runoff cells), bit-exact with
    the oracle."""
    net = syn.generate(syn.NetworkSpec(10_000, seed=23))
    tab = syn.runoff_mapping(net, (50, 80), seed=23, max_cells=9)
    cid = net.fields["catchment_id"]
    m = build_local_mapping(tab, cid, device)
    rp, col, w, _ = local_csr(tab, cid)
    assert np.diff(rp).max() > 4
    grid = syn.gridded_runoff((50, 80), 6, seed=2).astype(grid_dtype)
    got = apply_mapping(m, torch.as_tensor(grid, device=device), dtype=torch.float64,
                        unit_factor=86400000.0)
    ref = OF.map_grid(rp, col, w, grid.reshape(6, -1), unit_factor=86400000.0)
    np.testing.assert_array_equal(got.cpu().numpy(), ref)
