"""Parameter files: the reference's `parameters.nc` field set and axes.

The reference builds a model from one NetCDF file whose variables are the
module fields (cmfgpu/params/schema.py:14-140, written by
cmfgpu/params/merit_map.py:1085-1240) on named axes -- `catchment`,
`flood_level`, `bifurcation_path`, `bifurcation_level`, `levee`,
`reservoir`, `saved_points` -- plus map-construction metadata (grid size,
basin list, coordinates) that the routing does not read.

`FIELD_DIMS` restates the axes of every field the routing path reads.
`read_parameters` loads a file into a field dictionary (the argument of
`CaMaFlood(input_proxy=...)`) and checks each present field's axes and
shape against it; `write_parameters` writes one.  Two containers are read:

* NetCDF classic (CDF-1 / CDF-2 "64-bit offset"), through scipy;
* `.npz` archives with the same variable names (axes from FIELD_DIMS).

The reference writes NETCDF4, an HDF5 container, and no HDF5 reader is
available to this package; such a file is rejected with a message that names
the conversion (`nccopy -k 64-bit-offset`, or `xarray ... to_netcdf(format=
"NETCDF3_64BIT")`).  NetCDF classic has no 64-bit integer type, so identifier
fields are stored as int32 (or float64 when an id needs more than 31 bits)
and read back as int64.
"""
from __future__ import annotations

from pathlib import Path
from typing import Mapping

import numpy as np

# runtime size properties -> file axes (cmfgpu/params/schema.py:14-22)
MODEL_DIMENSIONS: dict[str, str] = {
    "num_catchments": "catchment",
    "num_output_catchments": "saved_points",
    "num_flood_levels": "flood_level",
    "num_bifurcation_paths": "bifurcation_path",
    "num_bifurcation_levels": "bifurcation_level",
    "num_levees": "levee",
    "num_reservoirs": "reservoir",
}

_C = ("catchment",)
_P = ("bifurcation_path",)
_PL = ("bifurcation_path", "bifurcation_level")
_LV = ("levee",)
_R = ("reservoir",)

# Axes of the fields the routing reads (the module fields of
# cmfgpu/modules/{base,bifurcation,levee,reservoir}.py).
FIELD_DIMS: dict[str, tuple[str, ...]] = {
    # base: topology and parameters
    "catchment_id": _C, "catchment_basin_id": _C, "downstream_id": _C,
    "river_width": _C, "river_length": _C, "river_height": _C, "catchment_elevation": _C,
    "catchment_area": _C, "downstream_distance": _C, "river_manning": _C, "flood_manning": _C,
    "flood_depth_table": ("catchment", "flood_level"),
    "output_catchment_id": ("saved_points",),
    # base: initial state
    "river_storage": _C, "flood_storage": _C, "protected_storage": _C, "protected_depth": _C,
    "river_depth": _C, "flood_depth": _C, "river_outflow": _C, "flood_outflow": _C,
    "river_cross_section_depth": _C, "flood_cross_section_depth": _C,
    "flood_cross_section_area": _C, "flood_fraction": _C,
    # bifurcation
    "bifurcation_path_id": _P, "bifurcation_catchment_id": _P, "bifurcation_downstream_id": _P,
    "bifurcation_manning": _PL, "bifurcation_width": _PL, "bifurcation_length": _P,
    "bifurcation_elevation": _PL, "bifurcation_outflow": _PL,
    "bifurcation_cross_section_depth": _PL,
    # levee
    "levee_id": _LV, "levee_catchment_id": _LV, "levee_crown_height": _LV, "levee_fraction": _LV,
    # reservoir
    "reservoir_id": _R, "reservoir_catchment_id": _R, "reservoir_capacity": _R,
    "conservation_volume": _R, "emergency_volume": _R, "normal_outflow": _R,
    "flood_control_outflow": _R, "reservoir_area": _R, "reservoir_total_inflow": _C,
}

# fields the base module cannot do without (the reference's required set,
# less the map metadata)
REQUIRED_FIELDS = ("catchment_id", "downstream_id", "river_width", "river_length",
                   "river_height", "catchment_elevation", "catchment_area",
                   "downstream_distance", "flood_depth_table")

# storage fields are fp64 in the model (the reference's "hpfloat")
HPFLOAT_FIELDS = frozenset({"river_storage", "flood_storage", "protected_storage",
                            "reservoir_total_inflow"})

ID_FIELDS = frozenset({k for k in FIELD_DIMS if k.endswith("_id")})


def _container(path: Path) -> str:
    with open(path, "rb") as fh:
        head = fh.read(8)
    if head[:3] == b"CDF" and head[3:4] in (b"\x01", b"\x02"):
        return "netcdf-classic"
    if head[:3] == b"CDF" and head[3:4] == b"\x05":
        return "netcdf-cdf5"
    if head[:8] == b"\x89HDF\r\n\x1a\n":
        return "hdf5"
    if head[:2] == b"PK":
        return "npz"
    return "unknown"


def check_fields(fields: Mapping[str, np.ndarray], dims: Mapping[str, tuple[str, ...]] | None = None) -> dict[str, int]:
    """Check every known field's rank, and that each axis has one length
    across all fields; returns the axis lengths.  `dims` gives the axes a
    file recorded (defaults to FIELD_DIMS)."""
    sizes: dict[str, int] = {}
    for name, arr in fields.items():
        if name not in FIELD_DIMS:
            continue
        want = FIELD_DIMS[name]
        got = tuple(dims[name]) if dims is not None and name in dims else want
        if got != want:
            raise ValueError(f"{name}: axes {got}, expected {want}")
        a = np.asarray(arr)
        if a.ndim != len(want):
            raise ValueError(f"{name}: rank {a.ndim}, expected {len(want)} ({', '.join(want)})")
        for ax, n in zip(want, a.shape):
            if sizes.setdefault(ax, int(n)) != int(n):
                raise ValueError(f"axis {ax!r} has length {sizes[ax]} and {n} ({name})")
    missing = [k for k in REQUIRED_FIELDS if k not in fields]
    if missing:
        raise ValueError(f"missing required fields: {missing}")
    return sizes


def read_parameters(path: str | Path) -> dict[str, np.ndarray]:
    """Field dictionary of a parameter file (see the module docstring)."""
    path = Path(path)
    kind = _container(path)
    dims: dict[str, tuple[str, ...]] = {}
    if kind == "netcdf-classic":
        from scipy.io import netcdf_file
        out = {}
        with netcdf_file(str(path), "r", mmap=False) as nc:
            for name, var in nc.variables.items():
                a = np.array(var.data, copy=True)
                dims[name] = tuple(var.dimensions)
                out[name] = a
    elif kind == "npz":
        with np.load(path) as z:
            out = {k: z[k] for k in z.files}
    elif kind == "hdf5":
        raise ValueError(
            f"{path} is NETCDF4 (HDF5), which needs an HDF5 reader this package does not have; "
            "convert it to NetCDF classic (nccopy -k 64-bit-offset in.nc out.nc) or to .npz")
    elif kind == "netcdf-cdf5":
        raise ValueError(f"{path} is NetCDF CDF-5; convert it with nccopy -k 64-bit-offset")
    else:
        raise ValueError(f"{path}: not a NetCDF classic, NETCDF4 or .npz parameter file")
    for k in list(out):
        if k in ID_FIELDS:
            out[k] = np.asarray(out[k]).astype(np.int64)
        elif k in HPFLOAT_FIELDS:
            out[k] = np.asarray(out[k], dtype=np.float64)
    check_fields(out, dims or None)
    return out


def write_parameters(path: str | Path, fields: Mapping[str, np.ndarray]) -> None:
    """Write the known fields of `fields` as NetCDF classic (64-bit offset)
    with the reference's axis names; other entries are skipped."""
    from scipy.io import netcdf_file
    known = {k: np.asarray(v) for k, v in fields.items() if k in FIELD_DIMS}
    sizes = check_fields(known)
    with netcdf_file(str(path), "w", version=2) as nc:
        for ax, n in sizes.items():
            nc.createDimension(ax, n)
        for name, a in known.items():
            if name in ID_FIELDS:
                a = a.astype(np.int64)
                fits = a.size == 0 or (a.min() >= -2**31 and a.max() < 2**31)
                a = a.astype(np.int32) if fits else a.astype(np.float64)
            elif a.dtype == np.bool_:
                a = a.astype(np.int8)
            elif a.dtype.kind == "i" and a.dtype.itemsize == 8:
                a = a.astype(np.int32)
            v = nc.createVariable(name, a.dtype, FIELD_DIMS[name])
            v[...] = a
