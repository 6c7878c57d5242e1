"""Drive the reference CUDA launchers (oracle/_ref) -- TEST INFRASTRUCTURE.

Runs the UNMODIFIED reference kernels (cmfgpu/phys/cuda, compiled by
oracle/build_ref.py) on the GPU in the reference's phase order
(cmfgpu/models/cama_flood_model.py:104-173), on inputs prepared by
oracle.reference_fields().  It is the GPU-side parity oracle and the source of
the committed golden fixtures; it is never part of the product path.
"""
from __future__ import annotations

import importlib.machinery
import importlib.util
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
_mod = None


def available() -> bool:
    return any((HERE / "_ref").glob("cmf_refcuda*.so"))


def module():
    global _mod
    if _mod is None:
        hits = sorted((HERE / "_ref").glob("cmf_refcuda*.so"))
        if not hits:
            raise RuntimeError("oracle/_ref/cmf_refcuda.so is not built (python oracle/build_ref.py)")
        loader = importlib.machinery.ExtensionFileLoader("cmf_refcuda", str(hits[0]))
        spec = importlib.util.spec_from_loader("cmf_refcuda", loader)
        _mod = importlib.util.module_from_spec(spec)
        loader.exec_module(_mod)
    return _mod


class RefCuda:
    """Reference kernels on CUDA tensors; the reference's own step order."""

    def __init__(self, fields: dict, modules, precision: str = "float32", device="cuda",
                 gravity: float = 9.8, min_kinematic_slope: float = 1e-5,
                 adaptive_time_factor: float = 0.7, block_size: int = 256):
        self.m = module()
        self.dev = torch.device(device)
        self.real = torch.float32 if precision == "float32" else torch.float64
        self.mods = set(modules)
        self.g = gravity
        self.min_kin = min_kinematic_slope
        self.alpha = adaptive_time_factor
        self.block = block_size
        t = {}
        for k, v in fields.items():
            a = np.asarray(v)
            if a.dtype == np.bool_:
                t[k] = torch.as_tensor(a).to(self.dev)
            elif k.endswith("_idx"):
                t[k] = torch.as_tensor(a.astype(np.int32)).to(self.dev)
            elif a.dtype == np.float64 and k in ("river_storage", "flood_storage",
                                                  "protected_storage", "reservoir_total_inflow"):
                t[k] = torch.as_tensor(a.copy()).to(self.dev)
            elif a.dtype.kind == "f":
                t[k] = torch.as_tensor(a.copy()).to(self.real).to(self.dev)
            else:
                t[k] = torch.as_tensor(a).to(self.dev)
        n = int(t["downstream_idx"].shape[0])
        self.n = n
        z64 = lambda: torch.zeros(n, dtype=torch.float64, device=self.dev)
        zr = lambda: torch.zeros(n, dtype=self.real, device=self.dev)
        for k in ("river_inflow", "flood_inflow", "outgoing_storage", "total_storage",
                  "global_bifurcation_outflow"):
            t.setdefault(k, z64())
        for k in ("limit_rate", "water_surface_elevation", "protected_water_surface_elevation",
                  "runoff"):
            t.setdefault(k, zr())
        t["time_step"] = torch.zeros(1, dtype=self.real, device=self.dev)
        t["outer_time_step"] = torch.zeros(1, dtype=self.real, device=self.dev)
        t["max_sub_steps"] = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.t = t

    def set_runoff(self, runoff) -> None:
        self.t["runoff"].copy_(torch.as_tensor(np.asarray(runoff)).to(self.real))

    def _opt(self, k, cond):
        return self.t[k] if cond else None

    def outflow(self):
        t, mods = self.t, self.mods
        bif, lev, res = "bifurcation" in mods, "levee" in mods, "reservoir" in mods
        self.m.launch_outflow(
            t["downstream_idx"], t["river_inflow"], t["river_outflow"], t["river_manning"],
            t["river_depth"], t["river_width"], t["river_length"], t["river_height"],
            t["river_storage"], t["flood_inflow"], t["flood_outflow"], t["flood_manning"],
            t["flood_depth"], t["protected_depth"], self._opt("is_levee", lev),
            t["catchment_elevation"], t["downstream_distance"], t["flood_storage"],
            t["protected_storage"], t["river_cross_section_depth"],
            t["flood_cross_section_depth"], t["flood_cross_section_area"],
            self._opt("global_bifurcation_outflow", bif), self._opt("total_storage", bif or res),
            t["outgoing_storage"], self._opt("water_surface_elevation", bif),
            self._opt("protected_water_surface_elevation", bif and lev),
            self.g, t["time_step"], self.n, bif, bif or res, bif, bif and lev, lev,
            self._opt("is_dam_upstream", res), res, self.min_kin, None, None, False, 0, self.block)

    def reservoir(self):
        t = self.t
        self.m.launch_reservoir_outflow(
            t["reservoir_catchment_idx"], t["downstream_idx"], t["reservoir_total_inflow"],
            t["river_outflow"], t["flood_outflow"], t["river_storage"], t["flood_storage"],
            t["conservation_volume"], t["emergency_volume"], t["adjustment_volume"],
            t["effective_normal_outflow"], t["adjustment_outflow"], t["flood_control_outflow"],
            t["runoff"], t["total_storage"], t["outgoing_storage"], t["time_step"], self.n,
            int(t["reservoir_catchment_idx"].shape[0]), self.block)

    def bif_outflow(self):
        t = self.t
        P, L = t["bifurcation_width"].shape
        if "levee" in self.mods:
            self.m.launch_levee_bif_outflow(
                t["bifurcation_catchment_idx"], t["bifurcation_downstream_idx"],
                t["bifurcation_manning"], t["bifurcation_outflow"], t["bifurcation_width"],
                t["bifurcation_length"], t["bifurcation_elevation"],
                t["bifurcation_cross_section_depth"], t["water_surface_elevation"],
                t["protected_water_surface_elevation"], t["total_storage"],
                t["outgoing_storage"], self.g, t["time_step"], self.n, int(P), int(L), self.block)
        else:
            self.m.launch_bif_outflow(
                t["bifurcation_catchment_idx"], t["bifurcation_downstream_idx"],
                t["bifurcation_manning"], t["bifurcation_outflow"], t["bifurcation_width"],
                t["bifurcation_length"], t["bifurcation_elevation"],
                t["bifurcation_cross_section_depth"], t["water_surface_elevation"],
                t["total_storage"], t["outgoing_storage"], self.g, t["time_step"], self.n,
                int(P), int(L), self.block)

    def inflow(self):
        t, mods = self.t, self.mods
        bif, res = "bifurcation" in mods, "reservoir" in mods
        self.m.launch_inflow(
            t["downstream_idx"], t["river_outflow"], t["flood_outflow"], t["river_storage"],
            t["flood_storage"], t["outgoing_storage"], t["river_inflow"], t["flood_inflow"],
            self._opt("limit_rate", bif), self._opt("reservoir_total_inflow", res),
            self._opt("is_reservoir", res), self.n, bif, res, self.block)

    def bif_inflow(self):
        t = self.t
        P, L = t["bifurcation_width"].shape
        self.m.launch_bif_inflow(
            t["bifurcation_catchment_idx"], t["bifurcation_downstream_idx"], t["limit_rate"],
            t["bifurcation_outflow"], t["global_bifurcation_outflow"], self.n, int(P), int(L),
            self.block)

    def flood_stage(self):
        t = self.t
        bif = "bifurcation" in self.mods
        self.m.launch_flood_stage(
            t["river_inflow"], t["flood_inflow"], t["river_outflow"], t["flood_outflow"],
            self._opt("global_bifurcation_outflow", bif), t["runoff"], None, None,
            t["time_step"], t["outgoing_storage"], t["river_storage"], t["flood_storage"],
            t["protected_storage"], t["river_depth"], t["flood_depth"], t["protected_depth"],
            t["flood_fraction"], t["river_height"], t["flood_depth_table"], t["catchment_area"],
            t["river_width"], t["river_length"], self.n, 0,
            int(t["flood_depth_table"].shape[-1]), bif, False, self.block)

    def levee_stage(self):
        t = self.t
        self.m.launch_levee_stage(
            t["levee_catchment_idx"], t["river_storage"], t["flood_storage"],
            t["protected_storage"], t["river_depth"], t["flood_depth"], t["protected_depth"],
            t["river_height"], t["flood_depth_table"], t["catchment_area"], t["river_width"],
            t["river_length"], t["levee_base_height"], t["levee_crown_height"],
            t["levee_fraction"], t["flood_fraction"], self.n,
            int(t["levee_catchment_idx"].shape[0]), int(t["flood_depth_table"].shape[-1]),
            self.block)

    def adaptive_sub_steps(self, outer_seconds: float) -> int:
        t = self.t
        t["outer_time_step"].fill_(outer_seconds)
        t["max_sub_steps"].zero_()
        self.m.launch_adaptive_time(
            t["river_depth"], t["downstream_distance"],
            self._opt("is_dam_related", "reservoir" in self.mods), t["max_sub_steps"],
            t["outer_time_step"], self.alpha, self.g, self.n, "reservoir" in self.mods, self.block)
        return int(t["max_sub_steps"].item())

    def substep(self):
        mods = self.mods
        self.outflow()
        if "reservoir" in mods:
            self.reservoir()
        if "bifurcation" in mods:
            self.bif_outflow()
        self.inflow()
        if "bifurcation" in mods:
            self.bif_inflow()
        self.flood_stage()
        if "levee" in mods:
            self.levee_stage()

    def step_advance(self, outer_seconds: float, adaptive: bool = True, fixed_n: int = 0) -> int:
        if adaptive:
            n = self.adaptive_sub_steps(outer_seconds)
        else:
            self.t["outer_time_step"].fill_(outer_seconds)
            n = int(fixed_n)
        self.t["time_step"].fill_(outer_seconds / n)
        for _ in range(n):
            self.substep()
        return n

    def state(self) -> dict[str, np.ndarray]:
        return {k: v.detach().cpu().numpy() for k, v in self.t.items()}
