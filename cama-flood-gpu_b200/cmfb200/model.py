"""CaMaFlood: the drop-in model object for the per-sub-step routing path.

Mirrors the reference controller (cmfgpu/models/cama_flood_model.py:46-173):
module objects `base`, `bifurcation`, `levee`, `reservoir`, `adaptive_time`,
`log` expose the reference's tensor names, dtypes and shapes;
`set_inputs(runoff)` stages forcing and `step_advance()` advances one forcing
interval in place.  All physics runs in libcmfb200 (hand-written sm_100a
kernels); this module only prepares tensors and calls the C ABI.

Catchment order.  Like the reference model, which reorders catchments when it
shards basins (partition_key / partition_group, cama_flood_model.py:59-60),
this model chooses its own catchment order: breadth-first from the river mouths
so that every catchment's upstream cells are contiguous.  `base.catchment_id`
is in model order; `to_model_order` / `to_input_order` convert arrays.
"""
from __future__ import annotations

import ctypes
import datetime as _dt
from types import SimpleNamespace
from typing import Iterable, Mapping, Optional

import numpy as np
import torch

from . import _lib, topology

REAL_BASE_PARAMS = ("river_width", "river_length", "river_height", "catchment_elevation",
                    "catchment_area", "downstream_distance", "river_manning", "flood_manning")
REAL_BASE_STATE = ("river_outflow", "flood_outflow", "river_depth", "flood_depth",
                   "protected_depth", "river_cross_section_depth", "flood_cross_section_depth",
                   "flood_cross_section_area", "flood_fraction")
STO_BASE_STATE = ("river_storage", "flood_storage", "protected_storage")
BATCHABLE = {
    "runoff": _lib.BATCH_RUNOFF,
    "river_manning": _lib.BATCH_RIVER_MANNING,
    "flood_manning": _lib.BATCH_FLOOD_MANNING,
    "river_width": _lib.BATCH_RIVER_WIDTH,
    "river_height": _lib.BATCH_RIVER_HEIGHT,
    "river_length": _lib.BATCH_RIVER_LENGTH,
}
KNOWN_MODULES = {"base", "adaptive_time", "bifurcation", "levee", "reservoir", "log"}


class Module(SimpleNamespace):
    """Attribute container standing in for a reference module (tensors by name)."""

    def tensors(self) -> dict[str, torch.Tensor]:
        return {k: v for k, v in vars(self).items() if isinstance(v, torch.Tensor)}


class InputProxy(dict):
    """Mapping of field name -> array, the role of hydroforge's InputProxy.

    `from_nc` reads a parameter file with the reference's field names and
    axes (cmfb200.params: NetCDF classic or .npz; NETCDF4/HDF5 is rejected
    with the conversion to use), `from_npz` an .npz of the same variables,
    `from_dict` wraps arrays already in memory."""

    @classmethod
    def from_nc(cls, path: str) -> "InputProxy":
        from .params import read_parameters
        return cls(read_parameters(path))

    @classmethod
    def from_dict(cls, fields: Mapping[str, np.ndarray]) -> "InputProxy":
        return cls({k: np.asarray(v) for k, v in fields.items()})

    @classmethod
    def from_npz(cls, path: str) -> "InputProxy":
        with np.load(path) as z:
            return cls({k: z[k] for k in z.files})


def _ids_to_index(catchment_id: np.ndarray, target_id: np.ndarray, self_on_missing: bool) -> np.ndarray:
    order = np.argsort(catchment_id, kind="stable")
    sorted_ids = catchment_id[order]
    pos = np.searchsorted(sorted_ids, target_id)
    pos_c = np.minimum(pos, sorted_ids.shape[0] - 1)
    found = sorted_ids[pos_c] == target_id
    idx = order[pos_c].astype(np.int64)
    if self_on_missing:
        idx = np.where(found, idx, np.arange(target_id.shape[0]))
    elif not found.all():
        raise ValueError(f"{int((~found).sum())} referenced catchment ids are not in catchment_id")
    return idx


def _require_positive(fields: Mapping[str, np.ndarray], names: Iterable[str]) -> None:
    bad = {n: int((~np.isfinite(fields[n]) | (fields[n] <= 0)).sum()) for n in names}
    bad = {k: v for k, v in bad.items() if v}
    if bad:
        details = ", ".join(f"{k}={v}" for k, v in bad.items())
        raise ValueError(
            "River geometry, catchment area, downstream distance, and Manning coefficients "
            f"must contain only finite values greater than zero; invalid element counts: {details}")


def validate_base(f: Mapping[str, np.ndarray]) -> None:
    """The reference's BaseModule validators (cmfgpu/modules/base.py:462-591)."""
    _require_positive(f, ("river_width", "river_length", "river_height", "catchment_area",
                          "downstream_distance", "river_manning", "flood_manning"))
    for name in ("catchment_elevation", "flood_depth_table"):
        if not np.isfinite(f[name]).all():
            raise ValueError("Elevation and flood-depth lookup values must be finite")
    if (f["flood_depth_table"] < 0).any():
        raise ValueError("flood_depth_table must be non-negative")
    for name in ("river_storage", "flood_storage", "protected_storage", "protected_depth",
                 "river_depth", "flood_depth", "river_cross_section_depth",
                 "flood_cross_section_depth", "flood_cross_section_area", "flood_fraction"):
        a = f[name]
        if (~np.isfinite(a) | (a < 0)).any():
            raise ValueError(
                "Initial storage, depth, and cross-section state must contain only finite "
                f"non-negative values (field {name})")
    if (f["flood_fraction"] > 1).any():
        raise ValueError("Initial flood_fraction must not exceed one")
    for name in ("river_outflow", "flood_outflow"):
        if not np.isfinite(f[name]).all():
            raise ValueError("Initial river and flood outflow must contain only finite values")
    tbl = f["flood_depth_table"]
    if tbl.shape[-1] > 1 and (np.diff(tbl, axis=-1) < 0).any():
        raise ValueError("flood_depth_table must be monotonically non-decreasing")


class CaMaFlood:
    """The routing model; one forcing interval per `step_advance()`.

    Parameters mirror the reference constructor where they apply:
    `opened_modules`, `BLOCK_SIZE`, and the module constants `gravity`,
    `min_kinematic_slope`, `adaptive_time_factor`.  Additions:
    `step_duration` (the forcing interval, seconds or timedelta),
    `precision` ("float32": fp32 fluxes + fp64 storage, the reference's mixed
    mode; "float64"), `num_members` (ensemble members, member-innermost),
    `batched_fields` (per-member parameters), `max_sub_step_seconds` (an
    optional CFL dt cap), `use_cuda_graph` and `budget` (fp64 water budget).
    `variables_to_save` takes the reference's form ({"mean": ["total_outflow"],
    "last": ["river_depth"]}, scripts/run_daily_bin.py:28) and accumulates
    those statistics on the device after every sub-step; `collect_statistics()`
    ends an output period (no file writer: the reference's NetCDF output
    workers are outside this path).
    """

    def __init__(self, device: str | torch.device = "cuda", input_proxy: Optional[Mapping] = None,
                 opened_modules: Iterable[str] = ("base",), step_duration=86400.0,
                 precision: str = "float32", num_members: int = 1,
                 batched_fields: Mapping[str, np.ndarray] | None = None,
                 BLOCK_SIZE: int = 256, use_cuda_graph: bool = True,
                 max_sub_step_seconds: float = 0.0, max_sub_steps_cap: int = 0,
                 gravity: float = 9.8, min_kinematic_slope: float = 1.0e-5,
                 adaptive_time_factor: float = 0.7, budget: bool = False,
                 variables_to_save: Optional[Mapping[str, Iterable[str]]] = None,
                 persistent: bool = False):
        if input_proxy is None:
            raise ValueError("input_proxy (field name -> array mapping) is required")
        mods = set(opened_modules) | {"base"}
        unknown = mods - KNOWN_MODULES
        if unknown:
            raise ValueError(f"unsupported modules {sorted(unknown)} (inflow and sea_level are "
                             "outside the routing path this model implements)")
        if precision not in ("float32", "float64"):
            raise ValueError("precision must be 'float32' (mixed) or 'float64'")
        self.device = torch.device(device)
        self.opened_modules = sorted(mods)
        if isinstance(step_duration, _dt.timedelta):
            step_duration = step_duration.total_seconds()
        self.step_seconds = float(step_duration)
        self.precision = precision
        self.real_np = np.float32 if precision == "float32" else np.float64
        self.real_torch = torch.float32 if precision == "float32" else torch.float64
        self.num_members = int(num_members)
        self.block_size = int(BLOCK_SIZE)
        self.use_cuda_graph = bool(use_cuda_graph)
        self.gravity = float(gravity)
        self.min_kinematic_slope = float(min_kinematic_slope)
        self.adaptive_time_factor = float(adaptive_time_factor)
        self.max_sub_step_seconds = float(max_sub_step_seconds)
        self.max_sub_steps_cap = int(max_sub_steps_cap)
        self.budget_enabled = bool(budget) or "log" in mods
        self.member_tile = 1
        self.persistent = False
        self._plan = None
        self._prepare(dict(input_proxy), dict(batched_fields or {}))
        self._upload()
        self._init_statistics(variables_to_save or {})
        self._create_plan()
        self.reset_statistics()
        if persistent:
            self.set_persistent(True)

    # ------------------------------------------------------------------ #
    # construction
    # ------------------------------------------------------------------ #
    @property
    def has(self):
        m = set(self.opened_modules)
        return SimpleNamespace(bif="bifurcation" in m, lev="levee" in m, res="reservoir" in m,
                               adaptive="adaptive_time" in m)

    def _prepare(self, f: dict, batched: dict) -> None:
        has = self.has
        cid = np.asarray(f["catchment_id"], dtype=np.int64)
        n = cid.shape[0]
        if "downstream_idx" in f:
            dn_in = np.asarray(f["downstream_idx"], dtype=np.int64)
            dn_in = np.where(dn_in < 0, np.arange(n), dn_in)
        else:
            dn_in = _ids_to_index(cid, np.asarray(f["downstream_id"], dtype=np.int64), True)
        base_in = {}
        for name in REAL_BASE_PARAMS:
            base_in[name] = np.asarray(f[name], dtype=self.real_np)
        base_in["flood_depth_table"] = np.asarray(f["flood_depth_table"], dtype=self.real_np)
        for name in REAL_BASE_STATE:
            base_in[name] = np.asarray(f.get(name, np.zeros(n)), dtype=self.real_np)
        for name in STO_BASE_STATE:
            base_in[name] = np.asarray(f.get(name, np.zeros(n)), dtype=np.float64)
        validate_base(base_in)

        order, up_ptr = topology.bfs_order(dn_in.astype(np.int32))
        inv = np.empty(n, dtype=np.int64)
        inv[order] = np.arange(n)
        self.order = order.astype(np.int64)       # model index -> input index
        self.inverse_order = inv                  # input index -> model index
        dn = inv[dn_in[order]].astype(np.int32)
        p = {k: np.ascontiguousarray(v[order]) for k, v in base_in.items()}
        p["catchment_id"] = cid[order]
        p["downstream_idx"] = dn
        p["upstream_ptr"] = up_ptr
        if "catchment_basin_id" in f:
            p["catchment_basin_id"] = np.asarray(f["catchment_basin_id"])[order]
        mouth = dn == np.arange(n)
        flags = np.where(mouth, _lib.CELL_MOUTH, 0).astype(np.uint8)
        levee_slot = np.full(n, -1, dtype=np.int32)
        res_slot = np.full(n, -1, dtype=np.int32)

        bif = {}
        if has.bif:
            ci = inv[_ids_to_index(cid, np.asarray(f["bifurcation_catchment_id"], dtype=np.int64), False)]
            di = inv[_ids_to_index(cid, np.asarray(f["bifurcation_downstream_id"], dtype=np.int64), False)]
            P = ci.shape[0]
            bif = {
                "bifurcation_path_id": np.asarray(f.get("bifurcation_path_id", np.arange(P))),
                "bifurcation_catchment_idx": ci.astype(np.int32),
                "bifurcation_downstream_idx": di.astype(np.int32),
                "bifurcation_manning": np.asarray(f["bifurcation_manning"], dtype=self.real_np),
                "bifurcation_width": np.asarray(f["bifurcation_width"], dtype=self.real_np),
                "bifurcation_length": np.asarray(f["bifurcation_length"], dtype=self.real_np),
                "bifurcation_elevation": np.array(f["bifurcation_elevation"], dtype=self.real_np),
                "bifurcation_outflow": np.asarray(f.get("bifurcation_outflow", np.zeros((P, 1))),
                                                  dtype=self.real_np),
                "bifurcation_cross_section_depth": np.asarray(
                    f.get("bifurcation_cross_section_depth", np.zeros((P, 1))), dtype=self.real_np),
            }
            L = bif["bifurcation_width"].shape[-1]
            for key in ("bifurcation_outflow", "bifurcation_cross_section_depth"):
                if bif[key].shape != (P, L):
                    bif[key] = np.zeros((P, L), dtype=self.real_np)
            if L > 8:
                raise ValueError("at most 8 bifurcation levels are supported")
            bptr, bpaths = topology.bifurcation_incidence(n, ci, di)
            bif["bif_cell_ptr"], bif["bif_cell_paths"] = bptr, bpaths
            flags |= np.where(np.diff(bptr) > 0, _lib.CELL_BIFURCATION, 0).astype(np.uint8)

        lev = {}
        if has.lev:
            lci = inv[_ids_to_index(cid, np.asarray(f["levee_catchment_id"], dtype=np.int64), False)]
            srt = np.argsort(lci, kind="stable")
            lci = lci[srt]
            if np.unique(lci).shape[0] != lci.shape[0]:
                raise ValueError("at most one levee per catchment")
            frac = np.asarray(f["levee_fraction"], dtype=self.real_np)[srt]
            crown = np.asarray(f["levee_crown_height"], dtype=self.real_np)[srt]
            if (~np.isfinite(frac) | (frac < 0) | (frac >= 1)).any():
                raise ValueError("levee_fraction must be finite and lie within [0, 1)")
            base_h = topology.levee_base_height(p["flood_depth_table"].astype(np.float32), lci,
                                                frac.astype(np.float32)).astype(self.real_np)
            bad = ~np.isfinite(crown) | ~np.isfinite(base_h) | (base_h >= crown)
            if bad.any():
                raise ValueError(f"{int(bad.sum())} levees have non-finite heights or a base "
                                 "height greater than or equal to the crown height")
            lev = {
                "levee_id": np.asarray(f.get("levee_id", np.arange(lci.shape[0])))[srt],
                "levee_catchment_idx": lci.astype(np.int32),
                "levee_crown_height": crown, "levee_fraction": frac,
                "levee_base_height": base_h,
            }
            flags[lci] |= _lib.CELL_LEVEE
            levee_slot[lci] = np.arange(lci.shape[0], dtype=np.int32)
        non_levee = (flags & _lib.CELL_LEVEE) == 0
        if (p["protected_storage"][non_levee] != 0).any():
            raise ValueError("protected_storage must be zero outside levee catchments")

        res = {}
        if has.res:
            rci = inv[_ids_to_index(cid, np.asarray(f["reservoir_catchment_id"], dtype=np.int64), False)]
            srt = np.argsort(rci, kind="stable")
            rci = rci[srt]
            if np.unique(rci).shape[0] != rci.shape[0]:
                raise ValueError("at most one reservoir per catchment")
            cons = np.asarray(f["conservation_volume"], dtype=np.float32)[srt]
            emerg = np.asarray(f["emergency_volume"], dtype=np.float32)[srt]
            cap = np.asarray(f["reservoir_capacity"], dtype=np.float32)[srt]
            if (emerg > cap).any():
                raise ValueError("Emergency volume exceeds reservoir capacity")
            if (cons > emerg).any():
                raise ValueError("Conservation volume exceeds emergency volume")
            qn = np.asarray(f["normal_outflow"], dtype=np.float32)[srt]
            qf = np.asarray(f["flood_control_outflow"], dtype=np.float32)[srt]
            der = topology.reservoir_derived(cons, emerg, qn, qf)
            is_res, related, upstream = topology.dam_masks(dn, rci)
            res = {
                "reservoir_id": np.asarray(f.get("reservoir_id", np.arange(rci.shape[0])))[srt],
                "reservoir_catchment_idx": rci.astype(np.int32),
                "reservoir_capacity": cap, "conservation_volume": cons, "emergency_volume": emerg,
                "normal_outflow": qn, "flood_control_outflow": qf,
                "reservoir_area": np.asarray(f.get("reservoir_area", np.zeros(rci.shape[0])),
                                             dtype=np.float32)[srt],
                **der,
                "is_reservoir": is_res, "is_dam_related": related, "is_dam_upstream": upstream,
            }
            rti = f.get("reservoir_total_inflow")
            res["reservoir_total_inflow"] = (np.zeros(n) if rti is None
                                             else np.asarray(rti, dtype=np.float64)[order])
            flags |= np.where(is_res, _lib.CELL_RESERVOIR, 0).astype(np.uint8)
            flags |= np.where(upstream, _lib.CELL_DAM_UPSTREAM, 0).astype(np.uint8)
            flags |= np.where(related, _lib.CELL_DAM_RELATED, 0).astype(np.uint8)
            res_slot[rci] = np.arange(rci.shape[0], dtype=np.int32)
            # cold start (reservoir.py:208-223) and dam-related path mask (:225-235)
            rs, fs = p["river_storage"], p["flood_storage"]
            upd = (rs[rci] + fs[rci]) < cons.astype(np.float64)
            rs[rci] = np.where(upd, cons.astype(np.float64), rs[rci])
            fs[rci] = np.where(upd, 0.0, fs[rci])
            self.dam_cells_initialized = int(upd.sum())
            if has.bif:
                masked = related[bif["bifurcation_catchment_idx"]] | related[bif["bifurcation_downstream_idx"]]
                bif["bifurcation_elevation"][masked, :] = self.real_np(1.0e20)
                self.bifurcation_paths_masked = int(masked.sum())
        p["cell_flags"] = flags
        p["levee_slot"] = levee_slot
        p["reservoir_slot"] = res_slot
        self._host = {"base": p, "bifurcation": bif, "levee": lev, "reservoir": res}
        self._batched_in = batched

    def _upload(self) -> None:
        dev, M, rt = self.device, self.num_members, self.real_torch
        has = self.has
        h = self._host
        p = h["base"]
        n = p["catchment_id"].shape[0]
        self.num_catchments = n

        def t(a, dtype=None):
            x = torch.as_tensor(np.ascontiguousarray(a))
            if dtype is not None:
                x = x.to(dtype)
            return x.to(dev).contiguous()

        def member(a, dtype):
            x = torch.as_tensor(np.ascontiguousarray(a)).to(dtype)
            if M > 1:
                x = x.unsqueeze(-1).expand(*x.shape, M).contiguous()
            return x.to(dev)

        base = Module()
        base.catchment_id = t(p["catchment_id"])
        base.downstream_idx = t(p["downstream_idx"], torch.int32)
        base.upstream_ptr = t(p["upstream_ptr"], torch.int32)
        base.cell_flags = t(p["cell_flags"], torch.uint8)
        base.levee_slot = t(p["levee_slot"], torch.int32)
        base.reservoir_slot = t(p["reservoir_slot"], torch.int32)
        self.batched_mask = 0
        for name in REAL_BASE_PARAMS:
            if name in self._batched_in:
                arr = np.asarray(self._batched_in[name], dtype=self.real_np)[self.order]
                if arr.shape != (n, M):
                    raise ValueError(f"batched field {name} must have shape (num_catchments, {M})")
                setattr(base, name, t(arr, rt))
                self.batched_mask |= BATCHABLE[name]
            else:
                setattr(base, name, t(p[name], rt))
        base.flood_depth_table = t(p["flood_depth_table"], rt)
        if "runoff" in self._batched_in or M > 1:
            base.runoff = torch.zeros((n, M) if M > 1 else (n,), dtype=rt, device=dev)
            if M > 1:
                self.batched_mask |= _lib.BATCH_RUNOFF
        else:
            base.runoff = torch.zeros(n, dtype=rt, device=dev)
        for name in REAL_BASE_STATE:
            setattr(base, name, member(p[name], rt))
        for name in STO_BASE_STATE:
            setattr(base, name, member(p[name], torch.float64))
        shape = (n, M) if M > 1 else (n,)
        base.river_inflow = torch.zeros(shape, dtype=torch.float64, device=dev)
        base.flood_inflow = torch.zeros(shape, dtype=torch.float64, device=dev)
        base.outgoing_storage = torch.zeros(shape, dtype=torch.float64, device=dev)
        base.total_storage = (torch.zeros(shape, dtype=torch.float64, device=dev)
                              if (has.bif or has.res) else None)
        base.water_surface_elevation = torch.zeros(shape, dtype=rt, device=dev) if has.bif else None
        base.protected_water_surface_elevation = (torch.zeros(shape, dtype=rt, device=dev)
                                                  if (has.bif and has.lev) else None)
        base.time_step = torch.zeros(M, dtype=rt, device=dev)
        base.outer_time_step = torch.zeros(1, dtype=rt, device=dev)
        base.current_step = torch.zeros(1, dtype=torch.int32, device=dev)
        base.gravity = self.gravity
        base.min_kinematic_slope = self.min_kinematic_slope
        base.num_catchments = n
        base.num_flood_levels = int(p["flood_depth_table"].shape[-1])
        self.base = base

        self.adaptive_time = None
        at_steps = torch.zeros(M, dtype=torch.int32, device=dev)
        if has.adaptive:
            self.adaptive_time = Module(adaptive_time_factor=self.adaptive_time_factor,
                                        max_sub_steps=at_steps)
        self._max_sub_steps = at_steps

        self.bifurcation = None
        if has.bif:
            b = h["bifurcation"]
            bm = Module()
            for k in ("bifurcation_path_id",):
                setattr(bm, k, t(b[k]))
            for k in ("bifurcation_catchment_idx", "bifurcation_downstream_idx", "bif_cell_ptr",
                      "bif_cell_paths"):
                setattr(bm, k, t(b[k], torch.int32))
            for k in ("bifurcation_manning", "bifurcation_width", "bifurcation_length",
                      "bifurcation_elevation"):
                setattr(bm, k, t(b[k], rt))
            bm.bifurcation_outflow = member(b["bifurcation_outflow"], rt)
            bm.bifurcation_cross_section_depth = member(b["bifurcation_cross_section_depth"], rt)
            bm.global_bifurcation_outflow = torch.zeros(shape, dtype=torch.float64, device=dev)
            bm.limit_rate = torch.zeros(shape, dtype=rt, device=dev)
            bm.num_bifurcation_paths = int(b["bifurcation_catchment_idx"].shape[0])
            bm.num_bifurcation_levels = int(b["bifurcation_width"].shape[-1])
            self.bifurcation = bm

        self.levee = None
        if has.lev:
            lv = h["levee"]
            lm = Module()
            lm.levee_id = t(lv["levee_id"])
            lm.levee_catchment_idx = t(lv["levee_catchment_idx"], torch.int32)
            for k in ("levee_crown_height", "levee_fraction", "levee_base_height"):
                setattr(lm, k, t(lv[k], rt))
            is_levee = torch.zeros(n, dtype=torch.bool)
            is_levee[torch.as_tensor(lv["levee_catchment_idx"], dtype=torch.int64)] = True
            lm.is_levee = is_levee.to(dev)
            lm.num_levees = int(lv["levee_catchment_idx"].shape[0])
            self.levee = lm

        self.reservoir = None
        if has.res:
            r = h["reservoir"]
            rm = Module()
            rm.reservoir_id = t(r["reservoir_id"])
            rm.reservoir_catchment_idx = t(r["reservoir_catchment_idx"], torch.int32)
            for k in ("reservoir_capacity", "conservation_volume", "emergency_volume",
                      "normal_outflow", "flood_control_outflow", "reservoir_area", "flood_volume",
                      "adjustment_volume", "effective_normal_outflow", "adjustment_outflow"):
                setattr(rm, k, t(r[k], rt))
            for k in ("is_reservoir", "is_dam_related", "is_dam_upstream"):
                setattr(rm, k, t(r[k], torch.bool))
            rm.reservoir_total_inflow = member(r["reservoir_total_inflow"], torch.float64)
            rm.num_reservoirs = int(r["reservoir_catchment_idx"].shape[0])
            self.reservoir = rm

        self.log = None
        self._budget = torch.zeros(_lib.BUDGET_TERMS, dtype=torch.float64, device=dev)
        if self.budget_enabled:
            self.log = Module(budget=self._budget)
        self._status = torch.zeros(1, dtype=torch.int32, device=dev)

    def _features(self) -> int:
        # an opened module with nothing in it (a basin shard without paths,
        # levees or reservoirs) keeps its module object but runs no kernel
        # part: the plan is built without its feature
        has = self.has
        f = 0
        if has.bif and self.bifurcation.num_bifurcation_paths > 0:
            f |= _lib.FEAT_BIFURCATION
        if has.lev and self.levee.num_levees > 0:
            f |= _lib.FEAT_LEVEE
        if has.res and self.reservoir.num_reservoirs > 0:
            f |= _lib.FEAT_RESERVOIR
        if has.adaptive:
            f |= _lib.FEAT_ADAPTIVE
        if self.budget_enabled:
            f |= _lib.FEAT_BUDGET
        if self.precision == "float64":
            f |= _lib.FEAT_FP64
        if self.use_cuda_graph:
            f |= _lib.FEAT_GRAPH
        return f

    def _view(self) -> _lib.CmfView:
        v = _lib.CmfView()
        b = self.base
        v.abi_version = _lib.ABI_VERSION
        v.features = self._features()
        v.num_catchments = self.num_catchments
        v.num_members = self.num_members
        v.num_flood_levels = b.num_flood_levels
        v.batched_mask = self.batched_mask
        v.gravity = self.gravity
        v.min_kinematic_slope = self.min_kinematic_slope
        v.adaptive_time_factor = self.adaptive_time_factor
        v.max_sub_step_seconds = self.max_sub_step_seconds
        v.max_sub_steps_cap = self.max_sub_steps_cap
        v.block_size = self.block_size

        def ptr(x):
            return x.data_ptr() if isinstance(x, torch.Tensor) else None

        for name in ("downstream_idx", "upstream_ptr", "cell_flags", "levee_slot", "reservoir_slot",
                     "river_width", "river_length", "river_height", "catchment_elevation",
                     "catchment_area", "downstream_distance", "river_manning", "flood_manning",
                     "flood_depth_table", "runoff", *REAL_BASE_STATE, *STO_BASE_STATE,
                     "river_inflow", "flood_inflow", "outgoing_storage", "total_storage",
                     "water_surface_elevation", "protected_water_surface_elevation",
                     "time_step", "outer_time_step", "current_step"):
            setattr(v, name, ptr(getattr(b, name)))
        v.max_sub_steps = ptr(self._max_sub_steps)
        v.budget = ptr(self._budget)
        v.status = ptr(self._status)
        if self.bifurcation is not None:
            bm = self.bifurcation
            v.num_bifurcation_paths = bm.num_bifurcation_paths
            v.num_bifurcation_levels = bm.num_bifurcation_levels
            v.bif_cell_ptr = ptr(bm.bif_cell_ptr)
            v.bif_cell_paths = ptr(bm.bif_cell_paths)
            for name in ("bifurcation_catchment_idx", "bifurcation_downstream_idx",
                         "bifurcation_manning", "bifurcation_width", "bifurcation_length",
                         "bifurcation_elevation", "bifurcation_outflow",
                         "bifurcation_cross_section_depth", "global_bifurcation_outflow",
                         "limit_rate"):
                setattr(v, name, ptr(getattr(bm, name)))
        if self.levee is not None:
            lm = self.levee
            v.num_levees = lm.num_levees
            for name in ("levee_catchment_idx", "levee_crown_height", "levee_fraction",
                         "levee_base_height"):
                setattr(v, name, ptr(getattr(lm, name)))
        if self.reservoir is not None:
            rm = self.reservoir
            v.num_reservoirs = rm.num_reservoirs
            for name in ("reservoir_catchment_idx", "conservation_volume", "emergency_volume",
                         "adjustment_volume", "effective_normal_outflow", "adjustment_outflow",
                         "flood_control_outflow", "reservoir_total_inflow"):
                setattr(v, name, ptr(getattr(rm, name)))
        return v

    def _create_plan(self) -> None:
        lib = _lib.lib()
        if self.device.type != "cuda":
            raise RuntimeError("CaMaFlood runs on a CUDA device only (no CPU fallback)")
        view = self._view()
        size = ctypes.c_size_t(0)
        _lib.check(lib.cmf_workspace_size(ctypes.byref(view), ctypes.byref(size)), "workspace_size")
        self._workspace = torch.zeros(max(int(size.value), 256), dtype=torch.uint8, device=self.device)
        view.workspace = self._workspace.data_ptr()
        view.workspace_bytes = self._workspace.numel()
        self._view_struct = view
        plan = ctypes.c_void_p()
        _lib.check(lib.cmf_plan_create(ctypes.byref(view), ctypes.byref(plan)), "plan_create")
        self._plan = plan
        if self.member_tile != 1:
            _lib.check(lib.cmf_plan_set_member_tile(plan, self.member_tile), "plan_set_member_tile")
        self._attach_statistics()
        if self.persistent:
            _lib.check(lib.cmf_plan_set_persistent(plan, 1), "plan_set_persistent")

    # ------------------------------------------------------------------ #
    # output statistics (variables_to_save)
    # ------------------------------------------------------------------ #
    def _init_statistics(self, spec: Mapping[str, Iterable[str]]) -> None:
        items = []
        for op, names in spec.items():
            if op not in _lib.STAT_OPS:
                raise ValueError(f"statistic '{op}' is not supported (one of {sorted(_lib.STAT_OPS)})")
            for name in ([names] if isinstance(names, str) else list(names)):
                if name not in _lib.STAT_VARIABLES:
                    raise ValueError(f"variable '{name}' cannot be saved "
                                     f"(one of {sorted(_lib.STAT_VARIABLES)})")
                if name.startswith("protected") and not (self.has.lev and self.levee.num_levees > 0):
                    raise ValueError(f"'{name}' needs the levee module with at least one levee")
                if (name, op) not in items:
                    items.append((name, op))
        if len(items) > _lib.MAX_STATISTICS:
            raise ValueError(f"at most {_lib.MAX_STATISTICS} statistics")
        self._stats_spec = items
        shape = tuple(self.base.river_depth.shape)
        self._stats_out = {f"{n}_{o}": torch.zeros(shape, dtype=torch.float64, device=self.device)
                           for n, o in items}
        self._stats_weight = torch.zeros(self.num_members, dtype=torch.float64, device=self.device)

    def _attach_statistics(self) -> None:
        arr = (_lib.CmfStatistic * max(len(self._stats_spec), 1))()
        for q, (name, op) in enumerate(self._stats_spec):
            arr[q].variable = _lib.STAT_VARIABLES[name]
            arr[q].op = _lib.STAT_OPS[op]
            arr[q].out = self._stats_out[f"{name}_{op}"].data_ptr()
        _lib.check(_lib.lib().cmf_stats_attach(self._plan, len(self._stats_spec), arr,
                                               self._stats_weight.data_ptr()), "stats_attach")

    def set_variables_to_save(self, spec: Optional[Mapping[str, Iterable[str]]]) -> None:
        """Replace the saved statistics (None or {} saves none) and start a new
        output period; the interval graph is rebuilt on the next step."""
        self._init_statistics(spec or {})
        self._attach_statistics()
        self.reset_statistics()

    @property
    def variables_to_save(self) -> dict[str, list[str]]:
        out: dict[str, list[str]] = {}
        for name, op in self._stats_spec:
            out.setdefault(op, []).append(name)
        return out

    def reset_statistics(self) -> None:
        """Start an output period (MEAN -> 0, MAX -> -inf, MIN -> +inf)."""
        _lib.check(_lib.lib().cmf_stats_reset(self._plan, self._stream()), "stats_reset")

    def accumulate_statistics(self, k: int) -> None:
        """Fold sub-step k run through the per-phase entry points into the
        statistics (step_advance does this itself)."""
        _lib.check(_lib.lib().cmf_stats_accumulate(self._plan, self._stream(), int(k)),
                   "stats_accumulate")

    def collect_statistics(self, reset: bool = True) -> dict[str, torch.Tensor]:
        """End the output period: {"<variable>_<op>": fp64 device tensor in
        model order ([N] or [N, M])}, then start the next one."""
        _lib.check(_lib.lib().cmf_stats_finalize(self._plan, self._stream()), "stats_finalize")
        out = {k: v.clone() for k, v in self._stats_out.items()}
        if reset:
            self.reset_statistics()
        return out

    # ------------------------------------------------------------------ #
    # public API (cama_flood_model.py:74-173)
    # ------------------------------------------------------------------ #
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _order_index(self, inverse: bool) -> torch.Tensor:
        """Device index tensor of the catchment permutation (cached)."""
        key = "_inverse_dev" if inverse else "_order_dev"
        t = getattr(self, key, None)
        if t is None:
            t = torch.as_tensor(self.inverse_order if inverse else self.order, device=self.device)
            setattr(self, key, t)
        return t

    @torch.inference_mode()
    def set_inputs(self, runoff, inflow=None, sea_surface_elevation=None,
                   order: str = "model") -> None:
        """Stage forcing (cama_flood_model.py:74-102): runoff in m^3/s, [N] or
        [N, M].  `order` names the catchment order of `runoff`: "model" (the
        order of base.catchment_id, which a forcing map built from those ids
        produces) or "input" (the order of the catchment_id this model was
        built from -- the reference model's own order, when the fields came
        from it); "input" runoff is permuted on the device."""
        if inflow is not None or sea_surface_elevation is not None:
            raise ValueError("inflow / sea_level modules are not part of this model")
        if order not in ("model", "input"):
            raise ValueError("order must be 'model' or 'input'")
        src = torch.as_tensor(runoff)
        if order == "input":
            src = src.to(self.device, non_blocking=True).reshape(self.base.runoff.shape)
            src = src.index_select(0, self._order_index(False))
        self.base.runoff.copy_(src.reshape(self.base.runoff.shape), non_blocking=True)

    def read_state(self, names: Optional[Iterable[str]] = None,
                   order: str = "model") -> dict[str, torch.Tensor]:
        """Copies of state tensors (all of state_tensors() by default).  With
        order="input" the catchment fields are permuted back to the order of
        the catchment_id this model was built from; path fields keep their
        order."""
        if order not in ("model", "input"):
            raise ValueError("order must be 'model' or 'input'")
        st = self.state_tensors()
        out = {}
        for k in (list(st) if names is None else list(names)):
            v = st[k] if k in st else getattr(self.base, k)
            if order == "input" and not k.startswith("bifurcation_"):
                v = v.index_select(0, self._order_index(True))
            out[k] = v.clone()
        return out

    @torch.inference_mode()
    def step_advance(self, num_sub_steps: Optional[int] = None) -> None:
        """Advance one forcing interval (cama_flood_model.py:104-173)."""
        fixed = 0
        if self.adaptive_time is None:
            if not num_sub_steps:
                raise ValueError("num_sub_steps is required without the adaptive_time module")
            fixed = int(num_sub_steps)
        elif num_sub_steps:
            fixed = int(num_sub_steps)
        _lib.check(_lib.lib().cmf_step_interval(self._plan, self._stream(), self.step_seconds, fixed),
                   "step_interval")

    # per-phase entry points (parity / debugging)
    def compute_adaptive_time_step(self, outer_seconds: Optional[float] = None) -> None:
        _lib.check(_lib.lib().cmf_phase_cfl(self._plan, self._stream(),
                                            float(outer_seconds or self.step_seconds)), "phase_cfl")

    def set_fixed_time_step(self, num_sub_steps: int, outer_seconds: Optional[float] = None) -> None:
        _lib.check(_lib.lib().cmf_phase_fixed_dt(self._plan, self._stream(),
                                                 float(outer_seconds or self.step_seconds),
                                                 int(num_sub_steps)), "phase_fixed_dt")

    def compute_momentum(self, diag: bool = True) -> None:
        """outflow + reservoir release + bifurcation outflow of one sub-step."""
        _lib.check(_lib.lib().cmf_phase_momentum(self._plan, self._stream(), int(diag)),
                   "phase_momentum")

    def compute_stage(self, diag: bool = True) -> None:
        """limiter + inflow + bifurcation inflow + storage/flood/levee stage."""
        _lib.check(_lib.lib().cmf_phase_stage(self._plan, self._stream(), int(diag)), "phase_stage")

    # The reference's phase callables, in the order of its sub-step loop
    # (cmfgpu/models/cama_flood_model.py:134-162).  The kernels here fuse
    # several phases: the first callable of each fused group launches the
    # group and the others are no-ops, so that loop runs unchanged on this
    # model.  The groups are:
    #   compute_outflow        outflow, reservoir release, (levee) bifurcation outflow
    #   compute_flood_stage    inflow and limiter, bifurcation inflow, flood stage, levee stage
    # The inflow diagnostics (river_inflow, flood_inflow) are therefore written
    # by compute_flood_stage, not by compute_inflow.
    def compute_outflow(self) -> None:
        self.compute_momentum(diag=True)

    def compute_reservoir_outflow(self) -> None:
        """Part of compute_outflow."""

    def compute_bifurcation_outflow(self) -> None:
        """Part of compute_outflow."""

    def compute_levee_bifurcation_outflow(self) -> None:
        """Part of compute_outflow."""

    def compute_inflow(self) -> None:
        """Part of compute_flood_stage (the inflow is gathered there)."""

    def compute_bifurcation_inflow(self) -> None:
        """Part of compute_flood_stage."""

    def compute_flood_stage(self) -> None:
        self.compute_stage(diag=True)

    def compute_flood_stage_log(self) -> None:
        """compute_flood_stage with the water budget.  The reference's _log
        kernels add per-sub-step fp32 sums (x 1e-9) into log buffers indexed
        by the current step; here the fused stage kernel folds the same
        storage terms, in fp64 and in a fixed order, into per-CTA partials
        that flush_budget() (and every step_advance) reduces into
        log.budget.  Like the reference's, it needs the log module (or
        budget=True): without it there is no budget to write, and it raises."""
        if not self.budget_enabled:
            raise ValueError("compute_flood_stage_log needs the log module (or budget=True)")
        self.compute_stage(diag=True)

    def compute_levee_stage(self) -> None:
        """Part of compute_flood_stage."""

    def compute_levee_stage_log(self) -> None:
        """Part of compute_flood_stage_log (the levee re-partition conserves
        the cell's storage, so the budget needs no levee term); needs the
        log module like it."""
        if not self.budget_enabled:
            raise ValueError("compute_levee_stage_log needs the log module (or budget=True)")

    def launch_substep_kernel(self, k: int, part: int) -> None:
        """Launch one kernel of sub-step k directly (for per-kernel timing)."""
        _lib.check(_lib.lib().cmf_launch_substep(self._plan, self._stream(), int(k), int(part)),
                   "launch_substep")

    def _rebuild_plan(self, block_size: int) -> None:
        """Rebuild the plan (and its interval graph) with another CTA size;
        the state lives in the model tensors between intervals, so this is
        safe between two step_advance calls."""
        self.close()
        self.block_size = int(block_size)
        self._create_plan()

    def set_member_tile(self, width: int) -> None:
        """Members per thread of the member-batched kernels (a divisor of
        num_members; 1 for one member).  Results do not depend on it."""
        width = int(width)
        if width < 1 or self.num_members % width or (self.num_members == 1 and width != 1):
            raise ValueError(f"member tile {width} must divide num_members={self.num_members}")
        _lib.check(_lib.lib().cmf_plan_set_member_tile(self._plan, width), "plan_set_member_tile")
        self.member_tile = width

    def set_persistent(self, on: bool = True) -> None:
        """Run each interval's sub-steps in one persistent cooperative kernel
        (grid-wide barriers between the phases) instead of the interval
        graph; the results are the same.  It pays on small networks, where a
        sub-step is a few microseconds of work.  One member, no budget and no
        output statistics; raises otherwise."""
        rc = _lib.lib().cmf_plan_set_persistent(self._plan, 1 if on else 0)
        if rc == _lib.CMF_ERR_UNSUPPORTED:
            raise ValueError("the persistent interval kernel runs one member without budget or "
                             "output statistics")
        _lib.check(rc, "plan_set_persistent")
        self.persistent = bool(on)

    def autotune_block_size(self, candidates=None, sub_steps: int = 6,
                            cache_path: Optional[str] = None, tile_candidates=None) -> dict:
        """Measure the candidate CTA sizes (and, with several members, member
        tiles) on this network and keep the fastest
        (cmfb200.autotune.tune_block_size); the state is unchanged."""
        from .autotune import DEFAULT_CANDIDATES, tune_block_size
        return tune_block_size(self, candidates or DEFAULT_CANDIDATES, sub_steps,
                               cache_path=cache_path, tile_candidates=tile_candidates)

    def flush_budget(self) -> None:
        _lib.check(_lib.lib().cmf_budget_flush(self._plan, self._stream()), "budget_flush")

    def sub_step_counts(self) -> torch.Tensor:
        return self._max_sub_steps

    def status(self) -> int:
        return int(self._status.item())

    def check_status(self) -> None:
        s = self.status()
        if s & _lib.STATUS_NONFINITE:
            raise FloatingPointError("routing produced non-finite storage or discharge")
        if s & _lib.STATUS_SUBSTEP_CAP:
            raise RuntimeError("CFL asked for more sub-steps than max_sub_steps_cap")
        if s & _lib.STATUS_SYNC_TIMEOUT:
            raise RuntimeError("a grid barrier of the persistent interval kernel timed out")

    # ------------------------------------------------------------------ #
    # ordering helpers, state I/O
    # ------------------------------------------------------------------ #
    def to_model_order(self, x):
        return x[self.order] if isinstance(x, np.ndarray) else x[torch.as_tensor(self.order, device=x.device)]

    def to_input_order(self, x):
        if isinstance(x, np.ndarray):
            return x[self.inverse_order]
        return x[torch.as_tensor(self.inverse_order, device=x.device)]

    STATE_FIELDS = REAL_BASE_STATE + STO_BASE_STATE

    def state_tensors(self) -> dict[str, torch.Tensor]:
        out = {k: getattr(self.base, k) for k in self.STATE_FIELDS}
        if self.bifurcation is not None:
            out["bifurcation_outflow"] = self.bifurcation.bifurcation_outflow
            out["bifurcation_cross_section_depth"] = self.bifurcation.bifurcation_cross_section_depth
        if self.reservoir is not None:
            out["reservoir_total_inflow"] = self.reservoir.reservoir_total_inflow
        return out

    def save_state(self, path: str) -> None:
        """Checkpoint the state tensors (model order) with torch.save."""
        torch.save({k: v.detach().cpu() for k, v in self.state_tensors().items()}, path)

    def load_state(self, path: str) -> None:
        data = torch.load(path)
        for k, v in self.state_tensors().items():
            v.copy_(data[k].to(v.device))

    def export_fields(self) -> dict[str, np.ndarray]:
        """Host copy of every tensor the routing reads or writes, model order."""
        out = {}
        for mod in (self.base, self.bifurcation, self.levee, self.reservoir):
            if mod is None:
                continue
            for k, v in mod.tensors().items():
                out[k] = v.detach().cpu().numpy()
        return out

    def close(self) -> None:
        if self._plan:
            _lib.lib().cmf_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
