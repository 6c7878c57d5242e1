"""Python driver of the CPU oracle (oracle/liborc.so) -- TEST INFRASTRUCTURE.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module;
the product (cmfb200 / libcmfb200) never imports it.

`Oracle` holds host copies of every tensor the reference sub-step touches, in
whatever catchment order it is given (the reference kernels are index-based,
so the oracle normally runs in the generator's original topological order
while the product runs in its breadth-first order), and advances them with
the C restatement of the reference kernels (cmf_oracle_impl.h).

`reference_fields(fields, modules)` prepares model inputs the way the
reference model does at construction: downstream index from ids
(hydroforge ReferenceIndexField, cmfgpu/modules/base.py:323), levee base
height (cmfgpu/modules/levee.py:209-217), reservoir masks and derived volumes
(cmfgpu/modules/reservoir.py:129-206) and the reservoir cold start
(cmfgpu/modules/reservoir.py:208-235).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# CMF_ORACLE_FMA=1 selects the FMA-contracted build (see oracle/Makefile)
LIB = HERE / ("liborc_fma.so" if os.environ.get("CMF_ORACLE_FMA") == "1" else "liborc.so")
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "cama-flood-gpu_b200"))

from cmfb200 import topology  # noqa: E402  (derived-parameter helpers, golden-pinned)

_I32, _I64, _F64, _P = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p

POINTERS = (
    "downstream_idx", "is_levee", "is_reservoir", "is_dam_upstream", "is_dam_related",
    "river_width", "river_length", "river_height", "catchment_elevation", "catchment_area",
    "downstream_distance", "river_manning", "flood_manning", "flood_depth_table", "runoff",
    "river_outflow", "flood_outflow", "river_depth", "flood_depth", "protected_depth",
    "river_cross_section_depth", "flood_cross_section_depth", "flood_cross_section_area",
    "flood_fraction", "river_storage", "flood_storage", "protected_storage",
    "river_inflow", "flood_inflow", "outgoing_storage", "total_storage",
    "global_bifurcation_outflow", "limit_rate", "water_surface_elevation",
    "protected_water_surface_elevation",
    "bifurcation_catchment_idx", "bifurcation_downstream_idx",
    "bifurcation_manning", "bifurcation_width", "bifurcation_length", "bifurcation_elevation",
    "bifurcation_outflow", "bifurcation_cross_section_depth",
    "levee_catchment_idx", "levee_crown_height", "levee_fraction", "levee_base_height",
    "reservoir_catchment_idx", "conservation_volume", "emergency_volume", "adjustment_volume",
    "effective_normal_outflow", "adjustment_outflow", "flood_control_outflow",
    "reservoir_total_inflow",
)
INT_FIELDS = {"downstream_idx", "bifurcation_catchment_idx", "bifurcation_downstream_idx",
              "levee_catchment_idx", "reservoir_catchment_idx"}
MASK_FIELDS = {"is_levee", "is_reservoir", "is_dam_upstream", "is_dam_related"}
STO_FIELDS = {"river_storage", "flood_storage", "protected_storage", "river_inflow",
              "flood_inflow", "outgoing_storage", "total_storage", "global_bifurcation_outflow",
              "reservoir_total_inflow"}


def _struct(real):
    class OrcModel(ctypes.Structure):
        _fields_ = [
            ("n", _I64), ("n_paths", _I64), ("n_levees", _I64), ("n_res", _I64),
            ("n_flood_levels", _I32), ("n_bif_levels", _I32),
            ("has_bif", _I32), ("has_levee", _I32), ("has_res", _I32),
            ("has_total_storage", _I32), ("has_wse", _I32), ("has_pwse", _I32),
            ("gravity", _F64), ("min_kinematic_slope", _F64), ("adaptive_time_factor", _F64),
            ("time_step", real), ("outer_time_step", real),
        ] + [(name, _P) for name in POINTERS]
    return OrcModel


OrcModel_f32 = _struct(ctypes.c_float)
OrcModel_f64 = _struct(ctypes.c_double)

_lib = None


def build() -> Path:
    """Compile liborc.so with the committed Makefile if it is missing or stale."""
    src = [HERE / "cmf_oracle.c", HERE / "cmf_oracle_impl.h", HERE / "Makefile"]
    libs = [HERE / "liborc.so", HERE / "liborc_fma.so"]
    if any(not l.exists() or any(p.stat().st_mtime > l.stat().st_mtime for p in src) for l in libs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        h = ctypes.CDLL(str(LIB))
        for sfx, st in (("_f32", OrcModel_f32), ("_f64", OrcModel_f64)):
            getattr(h, "orc_model_size" + sfx).restype = ctypes.c_size_t
            assert getattr(h, "orc_model_size" + sfx)() == ctypes.sizeof(st), "OrcModel layout"
            for name in ("orc_outflow", "orc_inflow", "orc_flood_stage", "orc_bif_outflow",
                         "orc_bif_inflow", "orc_reservoir", "orc_levee_stage", "orc_levee_bif",
                         "orc_substep"):
                f = getattr(h, name + sfx)
                f.restype = None
                f.argtypes = [ctypes.POINTER(st)]
            f = getattr(h, "orc_adaptive_time" + sfx)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.POINTER(st), _F64]
            f = getattr(h, "orc_step_advance" + sfx)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.POINTER(st), _F64, ctypes.c_int, ctypes.c_int, _F64]
        h.orc_set_threads.argtypes = [ctypes.c_int]
        h.orc_max_threads.restype = ctypes.c_int
        _lib = h
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def reference_fields(fields: dict, modules, precision: str = "float32") -> dict:
    """Model inputs prepared as the reference model would, in input order."""
    real = np.float32 if precision == "float32" else np.float64
    f = {k: np.array(v) for k, v in fields.items()}
    cid = f["catchment_id"].astype(np.int64)
    n = cid.shape[0]
    pos = {int(c): i for i, c in enumerate(cid)} if n < 200_000 else None

    def to_idx(ids, self_missing=False):
        ids = np.asarray(ids, dtype=np.int64)
        if pos is not None:
            out = np.array([pos.get(int(x), -1) for x in ids], dtype=np.int64)
        else:
            srt = np.argsort(cid)
            p = np.searchsorted(cid[srt], ids).clip(0, n - 1)
            out = np.where(cid[srt][p] == ids, srt[p], -1)
        if self_missing:
            out = np.where(out < 0, np.arange(ids.shape[0]), out)
        return out

    out = {}
    out["downstream_idx"] = to_idx(f["downstream_id"], True).astype(np.int32)
    for k in ("river_width", "river_length", "river_height", "catchment_elevation",
              "catchment_area", "downstream_distance", "river_manning", "flood_manning",
              "flood_depth_table", "river_outflow", "flood_outflow", "river_depth", "flood_depth",
              "protected_depth", "river_cross_section_depth", "flood_cross_section_depth",
              "flood_cross_section_area", "flood_fraction"):
        out[k] = f[k].astype(real)
    for k in ("river_storage", "flood_storage", "protected_storage"):
        out[k] = f[k].astype(np.float64)
    mods = set(modules)
    if "bifurcation" in mods:
        out["bifurcation_catchment_idx"] = to_idx(f["bifurcation_catchment_id"]).astype(np.int32)
        out["bifurcation_downstream_idx"] = to_idx(f["bifurcation_downstream_id"]).astype(np.int32)
        for k in ("bifurcation_manning", "bifurcation_width", "bifurcation_length",
                  "bifurcation_elevation", "bifurcation_outflow", "bifurcation_cross_section_depth"):
            out[k] = f[k].astype(real)
    if "levee" in mods:
        lci = to_idx(f["levee_catchment_id"])
        out["levee_catchment_idx"] = lci.astype(np.int32)
        out["levee_crown_height"] = f["levee_crown_height"].astype(real)
        out["levee_fraction"] = f["levee_fraction"].astype(real)
        out["levee_base_height"] = topology.levee_base_height(
            f["flood_depth_table"], lci, f["levee_fraction"]).astype(real)
        m = np.zeros(n, dtype=bool)
        m[lci] = True
        out["is_levee"] = m
    if "reservoir" in mods:
        rci = to_idx(f["reservoir_catchment_id"])
        out["reservoir_catchment_idx"] = rci.astype(np.int32)
        der = topology.reservoir_derived(f["conservation_volume"], f["emergency_volume"],
                                         f["normal_outflow"], f["flood_control_outflow"])
        out["conservation_volume"] = f["conservation_volume"].astype(real)
        out["emergency_volume"] = f["emergency_volume"].astype(real)
        out["flood_control_outflow"] = f["flood_control_outflow"].astype(real)
        for k in ("adjustment_volume", "effective_normal_outflow", "adjustment_outflow"):
            out[k] = der[k].astype(real)
        is_res, related, upstream = topology.dam_masks(out["downstream_idx"], rci)
        out["is_reservoir"], out["is_dam_related"], out["is_dam_upstream"] = is_res, related, upstream
        rti = f.get("reservoir_total_inflow")
        out["reservoir_total_inflow"] = np.zeros(n) if rti is None else rti.astype(np.float64)
        rs, fs = out["river_storage"], out["flood_storage"]
        cons = f["conservation_volume"].astype(np.float32).astype(np.float64)
        upd = (rs[rci] + fs[rci]) < cons
        rs[rci] = np.where(upd, cons, rs[rci])
        fs[rci] = np.where(upd, 0.0, fs[rci])
        if "bifurcation" in mods:
            masked = related[out["bifurcation_catchment_idx"]] | related[out["bifurcation_downstream_idx"]]
            out["bifurcation_elevation"][masked, :] = real(1.0e20)
    return out


class Oracle:
    """Reference sub-step on the host; arrays are owned copies."""

    def __init__(self, fields: dict, modules, precision: str = "float32", gravity: float = 9.8,
                 min_kinematic_slope: float = 1e-5, adaptive_time_factor: float = 0.7):
        self.precision = precision
        self.real = np.float32 if precision == "float32" else np.float64
        self.sfx = "_f32" if precision == "float32" else "_f64"
        st = OrcModel_f32 if precision == "float32" else OrcModel_f64
        mods = set(modules)
        self.mods = mods
        n = int(fields["downstream_idx"].shape[0])
        self.n = n
        self.a: dict[str, np.ndarray] = {}
        for k in POINTERS:
            if k in fields:
                v = fields[k]
                if k in INT_FIELDS:
                    v = np.ascontiguousarray(v, dtype=np.int32)
                elif k in MASK_FIELDS:
                    v = np.ascontiguousarray(v, dtype=np.uint8)
                elif k in STO_FIELDS:
                    v = np.array(v, dtype=np.float64, copy=True)
                else:
                    v = np.array(v, dtype=self.real, copy=True)
                self.a[k] = v
        for k in ("river_inflow", "flood_inflow", "outgoing_storage", "total_storage",
                  "global_bifurcation_outflow"):
            self.a.setdefault(k, np.zeros(n, dtype=np.float64))
        for k in ("limit_rate", "water_surface_elevation", "protected_water_surface_elevation"):
            self.a.setdefault(k, np.zeros(n, dtype=self.real))
        self.a.setdefault("runoff", np.zeros(n, dtype=self.real))
        m = st()
        m.n = n
        m.n_flood_levels = int(self.a["flood_depth_table"].shape[-1])
        m.has_bif = int("bifurcation" in mods)
        m.has_levee = int("levee" in mods)
        m.has_res = int("reservoir" in mods)
        m.has_total_storage = int(bool({"bifurcation", "reservoir"} & mods))
        m.has_wse = int("bifurcation" in mods)
        m.has_pwse = int({"bifurcation", "levee"} <= mods)
        m.gravity = gravity
        m.min_kinematic_slope = min_kinematic_slope
        m.adaptive_time_factor = adaptive_time_factor
        if m.has_bif:
            m.n_paths = int(self.a["bifurcation_catchment_idx"].shape[0])
            m.n_bif_levels = int(self.a["bifurcation_width"].shape[-1])
        if m.has_levee:
            m.n_levees = int(self.a["levee_catchment_idx"].shape[0])
        if m.has_res:
            m.n_res = int(self.a["reservoir_catchment_idx"].shape[0])
        for k, v in self.a.items():
            setattr(m, k, v.ctypes.data)
        self.m = m
        self.lib = lib()

    def _call(self, name, *args):
        return getattr(self.lib, name + self.sfx)(ctypes.byref(self.m), *args)

    def set_runoff(self, runoff) -> None:
        self.a["runoff"][:] = np.asarray(runoff, dtype=self.real)

    def set_time_step(self, dt: float, outer: float | None = None) -> None:
        self.m.time_step = float(self.real(dt))
        if outer is not None:
            self.m.outer_time_step = float(self.real(outer))

    def adaptive_sub_steps(self, outer_seconds: float, max_dt: float = 0.0) -> int:
        self.m.outer_time_step = float(self.real(outer_seconds))
        return int(self._call("orc_adaptive_time", float(max_dt)))

    def substep(self) -> None:
        self._call("orc_substep")

    def phase(self, name: str) -> None:
        self._call("orc_" + name)

    def step_advance(self, outer_seconds: float, adaptive: bool = True, fixed_n: int = 0,
                     max_dt: float = 0.0) -> int:
        return int(self._call("orc_step_advance", float(outer_seconds), int(bool(adaptive)),
                              int(fixed_n), float(max_dt)))

    @property
    def time_step(self) -> float:
        return float(self.m.time_step)

    def state(self) -> dict[str, np.ndarray]:
        return {k: v.copy() for k, v in self.a.items()}
