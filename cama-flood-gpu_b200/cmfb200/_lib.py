"""ctypes binding of libcmfb200.so (the C ABI declared in include/cmfb200.h).

The shared library is the only compute path of this package: there is no CPU
or PyTorch fallback.  `lib()` raises if the library is missing or its ABI does
not match, so a broken build fails loudly instead of running something else.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("CMFB200_LIB", _HERE / "lib" / "libcmfb200.so"))

ABI_VERSION = 1

# return codes
CMF_OK = 0
CMF_ERR_ARG = 1
CMF_ERR_CUDA = 2
CMF_ERR_TIMEOUT = 3
CMF_ERR_NUMERIC = 4
CMF_ERR_UNSUPPORTED = 5

STATUS_NONFINITE = 1
STATUS_SUBSTEP_CAP = 2
STATUS_SYNC_TIMEOUT = 8

FEAT_BIFURCATION = 1
FEAT_LEVEE = 2
FEAT_RESERVOIR = 4
FEAT_ADAPTIVE = 8
FEAT_BUDGET = 16
FEAT_FP64 = 32
FEAT_GRAPH = 64

CELL_MOUTH = 1
CELL_LEVEE = 2
CELL_RESERVOIR = 4
CELL_DAM_UPSTREAM = 8
CELL_DAM_RELATED = 16
CELL_BIFURCATION = 32

BATCH_RUNOFF = 1
BATCH_RIVER_MANNING = 2
BATCH_FLOOD_MANNING = 4
BATCH_RIVER_WIDTH = 8
BATCH_RIVER_HEIGHT = 16
BATCH_RIVER_LENGTH = 32

PART_MOMENTUM = 1
PART_STAGE = 2
PART_END = 4
PART_LIMIT = 8
PART_LEVEE = 16

BUDGET_STORAGE_START = 0
BUDGET_STORAGE_END = 1
BUDGET_RUNOFF_IN = 2
BUDGET_MOUTH_OUT = 3
BUDGET_CLIP_GAIN = 4
BUDGET_SUBSTEPS = 5
BUDGET_TERMS = 6

_I32, _I64, _F64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
_P = ctypes.c_void_p

# Pointer fields of CmfView, in declaration order.
VIEW_POINTERS = (
    # topology
    "downstream_idx", "upstream_ptr", "cell_flags", "levee_slot", "reservoir_slot",
    "bif_cell_ptr", "bif_cell_paths",
    # base parameters
    "river_width", "river_length", "river_height", "catchment_elevation", "catchment_area",
    "downstream_distance", "river_manning", "flood_manning", "flood_depth_table", "runoff",
    # base state
    "river_outflow", "flood_outflow", "river_depth", "flood_depth", "protected_depth",
    "river_cross_section_depth", "flood_cross_section_depth", "flood_cross_section_area",
    "flood_fraction", "river_storage", "flood_storage", "protected_storage",
    # diagnostics
    "river_inflow", "flood_inflow", "outgoing_storage", "total_storage",
    "global_bifurcation_outflow", "limit_rate", "water_surface_elevation",
    "protected_water_surface_elevation",
    # bifurcation
    "bifurcation_catchment_idx", "bifurcation_downstream_idx", "bifurcation_manning",
    "bifurcation_width", "bifurcation_length", "bifurcation_elevation", "bifurcation_outflow",
    "bifurcation_cross_section_depth",
    # levee
    "levee_catchment_idx", "levee_crown_height", "levee_fraction", "levee_base_height",
    # reservoir
    "reservoir_catchment_idx", "conservation_volume", "emergency_volume", "adjustment_volume",
    "effective_normal_outflow", "adjustment_outflow", "flood_control_outflow",
    "reservoir_total_inflow",
    # time control
    "time_step", "outer_time_step", "max_sub_steps", "current_step",
    "budget", "status",
    "workspace",
)


class CmfView(ctypes.Structure):
    _fields_ = [
        ("abi_version", _I32),
        ("features", _I32),
        ("num_catchments", _I64),
        ("num_members", _I32),
        ("num_flood_levels", _I32),
        ("num_bifurcation_paths", _I64),
        ("num_bifurcation_levels", _I32),
        ("batched_mask", _I32),
        ("num_levees", _I64),
        ("num_reservoirs", _I64),
        ("gravity", _F64),
        ("min_kinematic_slope", _F64),
        ("adaptive_time_factor", _F64),
        ("max_sub_step_seconds", _F64),
        ("max_sub_steps_cap", _I32),
        ("block_size", _I32),
    ] + [(name, _P) for name in VIEW_POINTERS] + [("workspace_bytes", ctypes.c_size_t)]


# output statistics (variables_to_save)
STAT_VARIABLES = {
    "river_outflow": 0, "flood_outflow": 1, "total_outflow": 2, "river_depth": 3,
    "flood_depth": 4, "flood_fraction": 5, "protected_depth": 6, "river_storage": 7,
    "flood_storage": 8, "protected_storage": 9,
}
STAT_OPS = {"mean": 0, "max": 1, "min": 2, "last": 3}
MAX_STATISTICS = 16


class CmfStatistic(ctypes.Structure):
    _fields_ = [("variable", _I32), ("op", _I32), ("out", _P)]


class CmfError(RuntimeError):
    """A libcmfb200 entry point returned a non-zero status."""

    def __init__(self, code: int, what: str):
        msg = _lib_handle.cmf_status_string(code).decode() if _lib_handle else str(code)
        super().__init__(f"{what}: {msg} (code {code})")
        self.code = code


_lib_handle = None


def lib() -> ctypes.CDLL:
    """Load libcmfb200.so once; raise if it is absent or ABI-incompatible."""
    global _lib_handle
    if _lib_handle is not None:
        return _lib_handle
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"libcmfb200.so not found at {LIB_PATH}; build it with "
            "`python cama-flood-gpu_b200/build.py` (there is no fallback path)")
    h = ctypes.CDLL(str(LIB_PATH))
    h.cmf_abi_version.restype = ctypes.c_int
    h.cmf_status_string.restype = ctypes.c_char_p
    h.cmf_status_string.argtypes = [ctypes.c_int]
    h.cmf_view_size.restype = ctypes.c_size_t
    h.cmf_view_field_offsets.restype = ctypes.c_int
    h.cmf_view_field_offsets.argtypes = [ctypes.POINTER(_I64), ctypes.c_int]
    h.cmf_workspace_size.restype = ctypes.c_int
    h.cmf_workspace_size.argtypes = [ctypes.POINTER(CmfView), ctypes.POINTER(ctypes.c_size_t)]
    h.cmf_plan_create.restype = ctypes.c_int
    h.cmf_plan_create.argtypes = [ctypes.POINTER(CmfView), ctypes.POINTER(_P)]
    h.cmf_plan_destroy.restype = None
    h.cmf_plan_destroy.argtypes = [_P]
    h.cmf_plan_set_member_tile.restype = ctypes.c_int
    h.cmf_plan_set_member_tile.argtypes = [_P, _I32]
    h.cmf_plan_set_persistent.restype = ctypes.c_int
    h.cmf_plan_set_persistent.argtypes = [_P, ctypes.c_int]
    h.cmf_probe_barrier_timeout.restype = ctypes.c_int
    h.cmf_probe_barrier_timeout.argtypes = [_P, _P, _P, _I32]
    h.cmf_step_interval.restype = ctypes.c_int
    h.cmf_step_interval.argtypes = [_P, _P, _F64, _I32]
    h.cmf_phase_momentum.restype = ctypes.c_int
    h.cmf_phase_momentum.argtypes = [_P, _P, ctypes.c_int]
    h.cmf_phase_stage.restype = ctypes.c_int
    h.cmf_phase_stage.argtypes = [_P, _P, ctypes.c_int]
    h.cmf_phase_cfl.restype = ctypes.c_int
    h.cmf_phase_cfl.argtypes = [_P, _P, _F64]
    h.cmf_phase_fixed_dt.restype = ctypes.c_int
    h.cmf_phase_fixed_dt.argtypes = [_P, _P, _F64, _I32]
    h.cmf_launch_substep.restype = ctypes.c_int
    h.cmf_launch_substep.argtypes = [_P, _P, _I32, ctypes.c_int]
    h.cmf_substep_noalloc.restype = ctypes.c_int
    h.cmf_substep_noalloc.argtypes = [ctypes.POINTER(CmfView), _P, ctypes.c_int]
    h.cmf_budget_flush.restype = ctypes.c_int
    h.cmf_budget_flush.argtypes = [_P, _P]
    h.cmf_stats_attach.restype = ctypes.c_int
    h.cmf_stats_attach.argtypes = [_P, ctypes.c_int, ctypes.POINTER(CmfStatistic), _P]
    h.cmf_stats_reset.restype = ctypes.c_int
    h.cmf_stats_reset.argtypes = [_P, _P]
    h.cmf_stats_accumulate.restype = ctypes.c_int
    h.cmf_stats_accumulate.argtypes = [_P, _P, _I32]
    h.cmf_stats_finalize.restype = ctypes.c_int
    h.cmf_stats_finalize.argtypes = [_P, _P]
    for name, args in {
        "cmf_topo_topological_sort": [_I64, _P, _P, _P],
        "cmf_topo_upstream_csr": [_I64, _P, _P, _P],
        "cmf_topo_bfs_order": [_I64, _P, _P, _P],
        "cmf_topo_init_river_depth": [_I64, _P, _P, _P, _P, _P],
        "cmf_topo_accumulate_upstream": [_I64, _P, _P, _P],
        "cmf_topo_accumulate_downstream": [_I64, _P, _P, _P],
    }.items():
        f = getattr(h, name)
        f.restype = ctypes.c_int
        f.argtypes = args
    if h.cmf_abi_version() != ABI_VERSION:
        raise RuntimeError(f"libcmfb200 ABI {h.cmf_abi_version()} != expected {ABI_VERSION}")
    if h.cmf_view_size() != ctypes.sizeof(CmfView):
        raise RuntimeError("CmfView layout mismatch between Python and libcmfb200")
    _lib_handle = h
    return h


def check(code: int, what: str) -> None:
    if code != CMF_OK:
        raise CmfError(code, what)


def declared_symbols() -> list[str]:
    """Every function name declared in include/cmfb200.h."""
    import re
    header = Path(__file__).resolve().parents[2] / "include" / "cmfb200.h"
    text = header.read_text()
    return sorted(set(re.findall(r"\b(cmf_[a-z0-9_]+)\s*\(", text)))
