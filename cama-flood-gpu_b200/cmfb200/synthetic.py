"""Seeded synthetic river networks and runoff standing in for CaMa-Flood maps.

No CaMa map or runoff data ships with the reference, so every workload is a
seeded synthetic network with the shapes and value distributions of the
reference's global maps:

* catchments in topological order; a non-mouth cell's downstream cell is
  drawn from the next 1..200 cells (clipped to the last cell); 3 % of cells
  and the last cell are mouths;
* river length lognormal (median 8 km, sigma 0.5); unit-catchment area
  U(50, 500) km^2; upstream area accumulated along the tree;
  river width = clip(0.4 A^0.5, 10, 2000) m, bankfull height =
  clip(0.1 A^0.3, 0.5, 15) m with A the upstream area in km^2;
* bed elevation falls downstream by length x slope, slope lognormal
  (median 1e-4, sigma 1.0); mouths sit at U(0, 5) m;
* 10 floodplain depth layers with Exp(mean 0.5 m) increments;
* Manning 0.03 (river) / 0.10 (floodplain); downstream distance = river
  length, 10 km at mouths (cmfgpu/params/merit_map.py:152-155);
* initial river depth by the reference's cold-start rule
  (cmfgpu/params/utils.py:140-157), river storage = length x width x depth;
* optional bifurcation paths (cell i to a cell up to 500 positions further,
  5 levels, widths lognormal median 50 m, level elevations by the bifori
  convention of cmfgpu/params/utils.py:558-591), levees on a fraction of
  cells (crown U(0.5, 1.0) x top layer, position U(0.2, 0.8), invalid
  base >= crown levees dropped as cmfgpu/params/merit_map.py:1032-1054 does)
  and reservoirs at top-5 % upstream-area cells (capacity log-uniform
  1e7..1e10 m^3, the default 0.37 flood share of
  cmfgpu/params/estimate_dam_params.py:462-482,693-694, Qn = mean inflow,
  Qf = 2 Qn);
* daily runoff gamma(k=0.5, mean 2 mm/day) per cell in m^3/s.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import topology

BIF_MANNING_LEVELS = (0.03, 0.1, 0.1, 0.1, 0.1)  # cmfgpu/params/merit_map.py:479


@dataclass
class NetworkSpec:
    num_catchments: int
    seed: int = 0
    mouth_fraction: float = 0.03
    max_jump: int = 200
    num_flood_levels: int = 10
    bifurcation_paths: int = 0
    bifurcation_levels: int = 5
    bifurcation_max_jump: int = 500
    levee_fraction: float = 0.0
    reservoirs: int = 0
    slope_sigma: float = 1.0


@dataclass
class Network:
    spec: NetworkSpec
    fields: dict = field(default_factory=dict)
    info: dict = field(default_factory=dict)

    @property
    def num_catchments(self) -> int:
        return int(self.fields["catchment_id"].shape[0])

    @property
    def opened_modules(self) -> list[str]:
        mods = ["base", "adaptive_time"]
        if "bifurcation_catchment_id" in self.fields:
            mods.append("bifurcation")
        if "levee_catchment_id" in self.fields:
            mods.append("levee")
        if "reservoir_catchment_id" in self.fields:
            mods.append("reservoir")
        return mods


def generate(spec: NetworkSpec, topo=None) -> Network:
    """The seeded network of `spec`.  `topo` supplies the three integration
    helpers (accumulate_upstream, accumulate_downstream, init_river_depth);
    the default is cmfb200.topology, which runs them in libcmfb200.  A
    process that must not load the product library passes another module with
    the same functions and gets the same network bit for bit."""
    topo = topology if topo is None else topo
    rng = np.random.default_rng(spec.seed)
    n = int(spec.num_catchments)
    idx = np.arange(n, dtype=np.int64)
    jump = rng.integers(1, spec.max_jump + 1, size=n)
    dn = np.minimum(idx + jump, n - 1)
    mouth = rng.random(n) < spec.mouth_fraction
    mouth[-1] = True
    dn[mouth] = idx[mouth]
    dn = dn.astype(np.int32)

    rivlen = (8000.0 * np.exp(0.5 * rng.standard_normal(n))).astype(np.float32)
    unit_area_km2 = rng.uniform(50.0, 500.0, size=n)
    up_area_km2 = topo.accumulate_upstream(dn, unit_area_km2)
    rivwth = np.clip(0.4 * up_area_km2 ** 0.5, 10.0, 2000.0).astype(np.float32)
    rivhgt = np.clip(0.1 * up_area_km2 ** 0.3, 0.5, 15.0).astype(np.float32)
    slope = 1e-4 * np.exp(spec.slope_sigma * rng.standard_normal(n))
    drop = rivlen.astype(np.float64) * slope
    drop[mouth] = rng.uniform(0.0, 5.0, size=int(mouth.sum()))
    elevation = topo.accumulate_downstream(dn, drop).astype(np.float32)
    K = spec.num_flood_levels
    fldhgt = np.cumsum(rng.exponential(0.5, size=(n, K)), axis=1).astype(np.float32)
    nxtdst = rivlen.copy()
    nxtdst[mouth] = np.float32(10000.0)
    catchment_area = (unit_area_km2 * 1e6).astype(np.float32)

    river_depth = topo.init_river_depth(elevation, rivhgt, dn)
    river_storage = (rivlen * rivwth * river_depth).astype(np.float64)

    f: dict[str, np.ndarray] = {
        "catchment_id": idx.copy(),
        "downstream_id": dn.astype(np.int64),
        "catchment_basin_id": np.zeros(n, dtype=np.int64),
        "river_width": rivwth,
        "river_length": rivlen,
        "river_height": rivhgt,
        "catchment_elevation": elevation,
        "catchment_area": catchment_area,
        "downstream_distance": nxtdst,
        "river_manning": np.full(n, 0.03, dtype=np.float32),
        "flood_manning": np.full(n, 0.10, dtype=np.float32),
        "flood_depth_table": fldhgt,
        "river_storage": river_storage,
        "flood_storage": np.zeros(n, dtype=np.float64),
        "protected_storage": np.zeros(n, dtype=np.float64),
        "protected_depth": np.zeros(n, dtype=np.float32),
        "river_depth": river_depth,
        "flood_depth": np.zeros(n, dtype=np.float32),
        "river_outflow": np.zeros(n, dtype=np.float32),
        "flood_outflow": np.zeros(n, dtype=np.float32),
        "river_cross_section_depth": np.zeros(n, dtype=np.float32),
        "flood_cross_section_depth": np.zeros(n, dtype=np.float32),
        "flood_cross_section_area": np.zeros(n, dtype=np.float32),
        "flood_fraction": np.zeros(n, dtype=np.float32),
    }
    info = {"upstream_area_km2": up_area_km2, "unit_area_km2": unit_area_km2}

    if spec.bifurcation_paths > 0:
        P = int(spec.bifurcation_paths)
        L = int(spec.bifurcation_levels)
        src = rng.integers(0, n - 1, size=P)
        dst = np.minimum(src + rng.integers(1, spec.bifurcation_max_jump + 1, size=P), n - 1)
        width = (50.0 * np.exp(0.5 * rng.standard_normal((P, L)))).astype(np.float64)
        p_elv = np.minimum(elevation[src], elevation[dst]).astype(np.float64)
        w1 = width[:, 0]
        dph = np.maximum(np.log10(w1) * 2.5 - 4.0, 0.5)
        dph = np.minimum(dph, np.maximum(rivhgt[src], rivhgt[dst]).astype(np.float64))
        elv = np.empty((P, L), dtype=np.float64)
        elv[:, 0] = p_elv - dph
        for lv in range(1, L):
            elv[:, lv] = p_elv + (lv - 1.0)
        man = np.tile(np.asarray((BIF_MANNING_LEVELS + (0.1,) * L)[:L], dtype=np.float32), (P, 1))
        f.update({
            "bifurcation_path_id": np.arange(P, dtype=np.int64),
            "bifurcation_catchment_id": src.astype(np.int64),
            "bifurcation_downstream_id": dst.astype(np.int64),
            "bifurcation_manning": man,
            "bifurcation_width": width.astype(np.float32),
            "bifurcation_length": (8000.0 * np.exp(0.5 * rng.standard_normal(P))).astype(np.float32),
            "bifurcation_elevation": elv.astype(np.float32),
            "bifurcation_outflow": np.zeros((P, L), dtype=np.float32),
            "bifurcation_cross_section_depth": np.zeros((P, L), dtype=np.float32),
        })

    if spec.levee_fraction > 0:
        cand = np.sort(rng.choice(n, size=int(round(spec.levee_fraction * n)), replace=False))
        crown = (rng.uniform(0.5, 1.0, size=cand.shape[0]) * fldhgt[cand, K - 1]).astype(np.float32)
        frac = rng.uniform(0.2, 0.8, size=cand.shape[0]).astype(np.float32)
        base = topology.levee_base_height(fldhgt, cand, frac)
        keep = (np.isfinite(frac) & np.isfinite(base) & np.isfinite(crown) & (frac >= 0)
                & (frac < 1.0) & (base >= 0) & (base < crown))
        info["levees_dropped"] = int((~keep).sum())
        lv = cand[keep]
        f.update({
            "levee_id": np.arange(lv.shape[0], dtype=np.int64),
            "levee_catchment_id": lv.astype(np.int64),
            "levee_crown_height": crown[keep],
            "levee_fraction": frac[keep],
        })

    if spec.reservoirs > 0:
        thresh = np.quantile(up_area_km2, 0.95)
        cand = np.flatnonzero(up_area_km2 >= thresh)
        R = min(int(spec.reservoirs), cand.shape[0])
        cells = np.sort(rng.choice(cand, size=R, replace=False))
        cap = 10.0 ** rng.uniform(7.0, 10.0, size=R)
        fld_vol = cap * 0.37
        con_vol = cap - fld_vol
        eme_vol = con_vol + fld_vol * 0.95
        qn = 2.0e-3 * up_area_km2[cells] * 1e6 / 86400.0
        f.update({
            "reservoir_id": np.arange(R, dtype=np.int64),
            "reservoir_catchment_id": cells.astype(np.int64),
            "reservoir_capacity": cap.astype(np.float32),
            "conservation_volume": con_vol.astype(np.float32),
            "emergency_volume": eme_vol.astype(np.float32),
            "normal_outflow": qn.astype(np.float32),
            "flood_control_outflow": (2.0 * qn).astype(np.float32),
            "reservoir_area": (cap / 20.0).astype(np.float32),
            "reservoir_total_inflow": np.zeros(n, dtype=np.float64),
        })
    return Network(spec=spec, fields=f, info=info)


def daily_runoff(network: Network, day: int, seed: int | None = None) -> np.ndarray:
    """Runoff of one day in m^3/s per catchment (gamma k=0.5, mean 2 mm/day)."""
    s = network.spec.seed if seed is None else seed
    rng = np.random.default_rng([s, 7919, int(day)])
    mm = rng.gamma(0.5, 4.0, size=network.num_catchments)
    area = network.fields["catchment_area"].astype(np.float64)
    return (mm * 1e-3 * area / 86400.0).astype(np.float32)


def diurnal_profile(day: int, seed: int = 0, hours: int = 24) -> np.ndarray:
    """A random positive diurnal profile normalised to mean 1."""
    rng = np.random.default_rng([seed, 104729, int(day)])
    w = rng.gamma(2.0, 1.0, size=hours)
    return (w / w.mean()).astype(np.float32)


# The workloads of the benchmark definitions.  Parity tests use scaled-down
# versions with the same generator.
CONFIGS = {
    # plain method, CPU-runnable: 60k catchments, 30 days, dt cap 3600 s
    "plain_60k": dict(spec=NetworkSpec(60_000, seed=0), days=30, interval=86400.0,
                      max_sub_step_seconds=3600.0),
    # global-15min scale, full physics: 250k catchments, 365 days
    "full_250k": dict(spec=NetworkSpec(250_000, seed=1, bifurcation_paths=8_000,
                                       levee_fraction=0.2, reservoirs=500),
                      days=365, interval=86400.0, max_sub_step_seconds=0.0),
    # 3-arcmin scale roofline case: 6M catchments, full physics, hourly runoff
    "full_6m": dict(spec=NetworkSpec(6_000_000, seed=2, bifurcation_paths=200_000,
                                     levee_fraction=0.2, reservoirs=7_000),
                    days=10, interval=3600.0, max_sub_step_seconds=0.0),
    # the same physics at a third of the size: one sub-step touches ~410 MB,
    # above the 126 MB L2, while a multi-pass profiler capture stays small
    "full_2m": dict(spec=NetworkSpec(2_000_000, seed=2, bifurcation_paths=66_667,
                                     levee_fraction=0.2, reservoirs=2_333),
                    days=10, interval=3600.0, max_sub_step_seconds=0.0),
}


def generate_basins(num_basins: int, total_catchments: int, seed: int = 0,
                    min_size: int = 100, max_size: int = 200_000) -> Network:
    """Independent single-mouth basins of log-uniform size, concatenated.

    Sizes are drawn log-uniform in [min_size, max_size] and then scaled so that
    they sum to about `total_catchments` (the ensemble workload: 500 basins,
    ~6M catchments per member).  Each basin is one tree from `generate` with
    its last cell as the only mouth; ids and `catchment_basin_id` are offset
    per basin."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(min_size), np.log(max_size), size=num_basins))
    sizes = np.maximum(np.round(sizes * total_catchments / sizes.sum()), 2).astype(np.int64)
    parts = []
    offset = 0
    for b, size in enumerate(sizes):
        net = generate(NetworkSpec(int(size), seed=seed * 100_003 + b + 1, mouth_fraction=0.0))
        f = dict(net.fields)
        f["catchment_id"] = f["catchment_id"] + offset
        f["downstream_id"] = f["downstream_id"] + offset
        f["catchment_basin_id"] = np.full(int(size), b, dtype=np.int64)
        parts.append(f)
        offset += int(size)
    fields = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    spec = NetworkSpec(int(offset), seed=seed, mouth_fraction=0.0)
    return Network(spec=spec, fields=fields, info={"basin_sizes": sizes})


def ensemble_factors(num_catchments: int, members: int, seed: int = 0):
    """Per-member perturbations of the ensemble workload, member-innermost:
    a multiplicative lognormal(sigma 0.3) runoff factor per catchment and a
    uniform +-20 % river-Manning factor, both [N, M] float32."""
    rng = np.random.default_rng([seed, 31337])
    runoff = np.exp(0.3 * rng.standard_normal((num_catchments, members))).astype(np.float32)
    manning = rng.uniform(0.8, 1.2, size=(num_catchments, members)).astype(np.float32)
    return runoff, manning


def runoff_mapping(network: Network, grid_shape=(720, 1440), seed: int = 0, max_cells: int = 4,
                   extra_rows: int = 0) -> dict:
    """A runoff mapping table in the reference's `.npz` layout
    (cmfgpu/params/export_bin.py:955-983) for `network` on a ny x nx runoff
    grid: every catchment draws 1..max_cells cells of the 2x2 block (3x3 when
    max_cells > 4, up to 9) at its grid position (catchments sweep the grid in
    generator order, so neighbours in the river tree share nearby cells),
    weights split its area.  Rows are
    shuffled against the network order and `extra_rows` rows for catchments
    outside the network are added, as a global table seen by one domain."""
    rng = np.random.default_rng([seed, 271828])
    ids = np.asarray(network.fields["catchment_id"], dtype=np.int64)
    area = np.asarray(network.fields["catchment_area"], dtype=np.float64)
    n = ids.size + int(extra_rows)
    ny, nx = int(grid_shape[0]), int(grid_shape[1])
    G = ny * nx
    all_ids = np.concatenate([ids, ids.max(initial=-1) + 1 + np.arange(int(extra_rows))])
    all_area = np.concatenate([area, rng.uniform(5e7, 5e8, size=int(extra_rows))])
    base = (np.arange(n, dtype=np.int64) * G) // max(n, 1)
    bx, by = base % nx, base // nx
    cnt = rng.integers(1, max_cells + 1, size=n)
    side = 2 if max_cells <= 4 else 3                      # 2x2 block, or 3x3 for up to 9 cells
    if max_cells > side * side:
        raise ValueError("max_cells is at most 9")
    offs = np.array([[dx, dy] for dy in range(side) for dx in range(side)], dtype=np.int64)
    perm = np.argsort(rng.random((n, side * side)), axis=1)  # which block cells, in which order
    rows = np.repeat(np.arange(n), cnt)
    slot = np.arange(rows.size) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    o = offs[perm[rows, slot % (side * side)]]
    cx = np.minimum(bx[rows] + o[:, 0], nx - 1)
    cy = np.minimum(by[rows] + o[:, 1], ny - 1)
    frac = rng.gamma(2.0, 1.0, size=rows.size)
    frac /= np.bincount(rows, weights=frac, minlength=n)[rows]
    data = all_area[rows] * frac
    order = rng.permutation(n)                             # table row order
    lens = cnt[order]
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    starts = np.cumsum(cnt) - cnt
    take = np.repeat(starts[order], lens) + (np.arange(indptr[-1]) - np.repeat(indptr[:-1], lens))
    return {
        "catchment_ids": all_ids[order],
        "sparse_data": data[take],
        "sparse_indices": (cy * nx + cx)[take].astype(np.int64),
        "sparse_indptr": indptr,
        "matrix_shape": np.array([n, G], dtype=np.int64),
        "coord_lon": np.linspace(-180 + 180 / nx, 180 - 180 / nx, nx),
        "coord_lat": np.linspace(90 - 90 / ny, -90 + 90 / ny, ny),
    }


def gridded_runoff(grid_shape, steps: int, seed: int = 0, members: int = 0) -> np.ndarray:
    """Raw gridded runoff in mm/day (gamma k=0.5, mean 2 mm/day), float32
    [steps, ny, nx] (or [steps, members, ny, nx]); unit_factor 86400000 maps
    mm/day x m^2 to m^3/s, as in the reference's daily-bin runs."""
    rng = np.random.default_rng([seed, 161803])
    shape = (steps, members, *grid_shape) if members else (steps, *grid_shape)
    return rng.gamma(0.5, 4.0, size=shape).astype(np.float32)
