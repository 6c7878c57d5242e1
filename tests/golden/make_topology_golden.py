"""Generate tests/golden/topology_golden.npz from the REFERENCE's own code.

    python tests/golden/make_topology_golden.py

Runs only where the reference checkout exists (oracle/refroot.py locates it).  On seeded
synthetic networks it executes, unmodified:
  cmfgpu/params/utils.py   topological_sort, build_upstream_csr,
                           compute_init_river_depth (numba)
  cmfgpu/modules/levee.py  LeveeModule._interp_lookup (levee base height)
  cmfgpu/modules/reservoir.py  derived volumes / outflows and dam masks
and stores inputs and outputs.  tests/test_topology.py checks the native
topology code against them bit for bit.
"""
from __future__ import annotations

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1] / "cama-flood-gpu_b200"))

import _refimport as R  # noqa: E402
from cmfb200 import synthetic as syn  # noqa: E402


def main() -> None:
    u = R.load("cmfgpu.params.utils", "cmfgpu/params/utils.py")
    lv = R.load("cmfgpu.modules.levee", "cmfgpu/modules/levee.py")
    rs = R.load("cmfgpu.modules.reservoir", "cmfgpu/modules/reservoir.py")
    out = {}
    for case, (n, seed) in enumerate([(3000, 11), (2500, 12), (1200, 13)]):
        net = syn.generate(syn.NetworkSpec(n, seed=seed, levee_fraction=0.3, reservoirs=25))
        f = net.fields
        cid = f["catchment_id"]
        dn_idx = f["downstream_id"].astype(np.int64)
        mouth = dn_idx == np.arange(n)
        # shuffled ids and order for the topological sort
        rng = np.random.default_rng(seed)
        perm = rng.permutation(n)
        ids = rng.choice(10 * n, size=n, replace=False).astype(np.int64)
        sh_cid = ids[perm]
        sh_down = np.where(mouth[perm], -1, ids[dn_idx[perm]]).astype(np.int64)
        out[f"c{case}_topo_catchment_id"] = sh_cid
        out[f"c{case}_topo_downstream_id"] = sh_down
        out[f"c{case}_topo_order"] = np.asarray(u.topological_sort(sh_cid, sh_down))
        ptr, ind = u.build_upstream_csr(sh_cid, sh_down)
        out[f"c{case}_csr_indptr"], out[f"c{case}_csr_indices"] = np.asarray(ptr), np.asarray(ind)
        # initial depth in topological order (mouths -1, merit_map convention)
        dn_m1 = np.where(mouth, -1, dn_idx).astype(np.int64)
        ce = f["catchment_elevation"].astype(np.float32)
        rh = f["river_height"].astype(np.float32)
        out[f"c{case}_depth_downstream_idx"] = dn_m1
        out[f"c{case}_depth_elevation"] = ce
        out[f"c{case}_depth_river_height"] = rh
        out[f"c{case}_init_river_depth"] = np.asarray(u.compute_init_river_depth(ce, rh, dn_m1))
        # levee base height
        table = torch.as_tensor(f["flood_depth_table"].astype(np.float32))
        lci = torch.as_tensor(f["levee_catchment_id"].astype(np.int64))
        frac = torch.as_tensor(f["levee_fraction"].astype(np.float32))
        fake = SimpleNamespace(
            gather_tensor=lambda t, idx, batched=False: t[idx],
            levee_catchment_idx=lci,
            base=SimpleNamespace(is_batched=lambda k: False, num_flood_levels=table.shape[-1]))
        base_h = lv.LeveeModule._interp_lookup(fake, table, frac * table.shape[-1])
        out[f"c{case}_levee_table"] = table.numpy()
        out[f"c{case}_levee_catchment_idx"] = lci.numpy()
        out[f"c{case}_levee_fraction"] = frac.numpy()
        out[f"c{case}_levee_base_height"] = base_h.numpy()
        # reservoir derived parameters and masks
        R_ = rs.ReservoirModule.__dict__
        rv = SimpleNamespace(
            conservation_volume=torch.as_tensor(f["conservation_volume"]),
            emergency_volume=torch.as_tensor(f["emergency_volume"]),
            normal_outflow=torch.as_tensor(f["normal_outflow"]),
            flood_control_outflow=torch.as_tensor(f["flood_control_outflow"]))
        for name in ("flood_volume", "adjustment_volume", "effective_normal_outflow",
                     "adjustment_outflow"):
            setattr(rv, name, R_[name].func(rv))
            out[f"c{case}_res_{name}"] = getattr(rv, name).numpy()
        for name in ("conservation_volume", "emergency_volume", "normal_outflow",
                     "flood_control_outflow"):
            out[f"c{case}_res_{name}"] = f[name]
        dnt = torch.as_tensor(dn_idx)
        rci = torch.as_tensor(f["reservoir_catchment_id"].astype(np.int64))
        mv = SimpleNamespace(base=SimpleNamespace(downstream_idx=dnt, num_catchments=n,
                                                  catchment_id=torch.as_tensor(cid)),
                             reservoir_catchment_idx=rci)
        mv.is_reservoir = R_["is_reservoir"].func(mv)
        mv.is_dam_related = R_["is_dam_related"].func(mv)
        mv.is_dam_upstream = R_["is_dam_upstream"].func(mv)
        out[f"c{case}_res_downstream_idx"] = dn_idx
        out[f"c{case}_res_catchment_idx"] = rci.numpy()
        for name in ("is_reservoir", "is_dam_related", "is_dam_upstream"):
            out[f"c{case}_res_{name}"] = getattr(mv, name).numpy()
    path = HERE / "topology_golden.npz"
    np.savez_compressed(path, **out)
    print(path, path.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
