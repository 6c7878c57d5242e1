"""Runoff forcing map: gridded runoff -> catchment runoff on the GPU.

The step in front of the routing path.  The reference reads a runoff mapping
table (an `.npz` written by hydroforge's `generate_mapping_table`,
scripts/make_runoff_map.py), restricts it to the model's catchments with
`dataset.build_local_mapping(mapping_file, desired_catchment_ids, device)`
and maps every chunk of gridded runoff with
`dataset.shard_forcing(runoff_chunk.to(device), local_mapping)`
(scripts/run_daily_bin.py:98-118).  hydroforge (>= 0.1.0, the reference's
pyproject dependency) is not part of the reference tree; the table format
used here is the one the reference itself reads back in
cmfgpu/params/export_bin.py:955-983:

    catchment_ids  [R]        row -> catchment id
    sparse_data    [nnz]      weights (contributing area, m^2)
    sparse_indices [nnz]      column = flattened runoff-grid cell iy * nx + ix
                              (export_bin.py:1071-1075)
    sparse_indptr  [R + 1]    CSR row pointers
    matrix_shape   [2]        (R, ny * nx)
    coord_lon [nx], coord_lat [ny]

`build_local_mapping` returns a `RunoffMapping` whose rows follow
`desired_catchment_ids` (pass `model.base.catchment_id`, the model order) and
`shard_forcing` applies it with the `cmf_forcing_apply` kernel of
libcmfb200.so: out[t, r] = (sum_k w_k * grid[t, col_k]) * (1 / unit_factor),
summed in the table's entry order in fp64.  There is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path
from typing import Mapping, Optional, Union

import numpy as np
import torch

from . import _lib

MAPPING_KEYS = ("catchment_ids", "sparse_data", "sparse_indices", "sparse_indptr", "matrix_shape")

DTYPE_F32 = 0
DTYPE_F64 = 1
SKIP_MISSING = 1
CLAMP_NEGATIVE = 2
STATUS_BAD_INDEX = 4

_DTYPE_CODE = {torch.float32: DTYPE_F32, torch.float64: DTYPE_F64}


class CmfForcingMap(ctypes.Structure):
    _fields_ = [
        ("num_rows", ctypes.c_int64),
        ("num_cols", ctypes.c_int64),
        ("row_ptr", ctypes.c_void_p),
        ("col", ctypes.c_void_p),
        ("weight", ctypes.c_void_p),
    ]


def _bind(h: ctypes.CDLL) -> ctypes.CDLL:
    if getattr(h, "_forcing_bound", False):
        return h
    I, I32, I64, D, P = ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    h.cmf_forcing_apply.restype = I
    h.cmf_forcing_apply.argtypes = [ctypes.POINTER(CmfForcingMap), P, P, I, I32, I32, I64, I64,
                                    P, I, I64, I64, I64, D, D, I, P]
    h._forcing_bound = True
    return h


def load_mapping_table(mapping_file: Union[str, Path, Mapping]) -> dict:
    """Read a runoff mapping table (`.npz` path or an already-loaded mapping)."""
    if isinstance(mapping_file, Mapping):
        z = dict(mapping_file)
    else:
        with np.load(str(mapping_file)) as f:
            z = {k: f[k] for k in f.files}
    missing = [k for k in MAPPING_KEYS if k not in z]
    if missing:
        raise ValueError(f"runoff mapping table lacks {missing}")
    return z


def local_csr(table: Mapping, desired_catchment_ids: np.ndarray, allow_missing: bool = False):
    """Rows of `table` for `desired_catchment_ids`, in that order (host numpy).

    Returns (row_ptr int64 [n+1], col int32 [nnz], weight float64 [nnz],
    num_cols).  A desired catchment absent from the table raises unless
    `allow_missing`, in which case its row is empty (zero runoff)."""
    ids = np.asarray(table["catchment_ids"]).astype(np.int64).ravel()
    indptr = np.asarray(table["sparse_indptr"]).astype(np.int64).ravel()
    indices = np.asarray(table["sparse_indices"]).astype(np.int64).ravel()
    data = np.asarray(table["sparse_data"]).astype(np.float64).ravel()
    shape = tuple(int(x) for x in np.asarray(table["matrix_shape"]).ravel())
    if len(shape) != 2 or shape[0] != ids.size or indptr.size != ids.size + 1:
        raise ValueError("runoff mapping table: inconsistent catchment_ids / indptr / matrix_shape")
    if indptr[0] != 0 or np.any(np.diff(indptr) < 0) or indptr[-1] != indices.size or data.size != indices.size:
        raise ValueError("runoff mapping table: malformed CSR arrays")
    num_cols = shape[1]
    if "coord_lon" in table and "coord_lat" in table:
        nx, ny = np.asarray(table["coord_lon"]).size, np.asarray(table["coord_lat"]).size
        if nx * ny != num_cols:
            raise ValueError(f"runoff mapping table: matrix_shape[1]={num_cols} != {ny} x {nx} grid")
    if num_cols > np.iinfo(np.int32).max:
        raise ValueError("runoff grid larger than 2^31 cells")
    if indices.size and (indices.min() < 0 or indices.max() >= num_cols):
        raise ValueError("runoff mapping table: column index outside the grid")
    if np.unique(ids).size != ids.size:
        raise ValueError("runoff mapping table: duplicate catchment ids")

    want = np.asarray(desired_catchment_ids).astype(np.int64).ravel()
    order = np.argsort(ids, kind="stable")
    if ids.size:
        pos = np.minimum(np.searchsorted(ids[order], want), ids.size - 1)
        found = ids[order][pos] == want
    else:
        pos = np.zeros(want.size, dtype=np.int64)
        order = np.zeros(1, dtype=np.int64)
        found = np.zeros(want.size, dtype=bool)
    if not found.all() and not allow_missing:
        raise ValueError(f"{int((~found).sum())} desired catchment ids are not in the runoff mapping table")
    src = np.where(found, order[pos], -1)
    lens = np.where(found, indptr[np.maximum(src, 0) + 1] - indptr[np.maximum(src, 0)], 0)
    row_ptr = np.zeros(want.size + 1, dtype=np.int64)
    np.cumsum(lens, out=row_ptr[1:])
    nnz = int(row_ptr[-1])
    # entry e of output row r comes from table entry indptr[src[r]] + (e - row_ptr[r])
    rows = np.repeat(np.arange(want.size), lens)
    take = np.repeat(indptr[np.maximum(src, 0)], lens) + (np.arange(nnz) - row_ptr[rows])
    return row_ptr, indices[take].astype(np.int32), data[take], num_cols


@dataclass
class RunoffMapping:
    """A mapping table restricted to (and ordered like) a model's catchments,
    resident on the device."""
    row_ptr: torch.Tensor   # int64 [rows + 1]
    col: torch.Tensor       # int32 [nnz]
    weight: torch.Tensor    # float64 [nnz], m^2
    num_cols: int           # runoff grid cells
    grid_shape: Optional[tuple] = None  # (ny, nx) when the table names its coordinates
    catchment_id: Optional[np.ndarray] = None

    @property
    def num_rows(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def used_cells(self) -> int:
        """Distinct grid cells read per series."""
        return int(torch.unique(self.col).numel())

    def _c(self) -> CmfForcingMap:
        return CmfForcingMap(self.num_rows, self.num_cols, self.row_ptr.data_ptr(),
                             self.col.data_ptr(), self.weight.data_ptr())

    def bytes_per_launch(self, series: int, grid_itemsize: int = 4, out_itemsize: int = 4) -> int:
        """Algorithmic HBM bytes of one launch over `series` forcing steps x members."""
        return (8 * (self.num_rows + 1) + 12 * self.nnz
                + series * (self.used_cells() * grid_itemsize + self.num_rows * out_itemsize))


def build_local_mapping(mapping_file, desired_catchment_ids, device="cuda",
                        allow_missing: bool = False) -> RunoffMapping:
    """hydroforge `dataset.build_local_mapping` (scripts/run_daily_bin.py:98-102)."""
    table = load_mapping_table(mapping_file)
    row_ptr, col, weight, num_cols = local_csr(table, desired_catchment_ids, allow_missing)
    dev = torch.device(device)
    grid_shape = None
    if "coord_lon" in table and "coord_lat" in table:
        grid_shape = (int(np.asarray(table["coord_lat"]).size), int(np.asarray(table["coord_lon"]).size))
    return RunoffMapping(torch.as_tensor(row_ptr).to(dev), torch.as_tensor(col).to(dev),
                         torch.as_tensor(weight).to(dev), num_cols, grid_shape,
                         np.asarray(desired_catchment_ids).astype(np.int64).ravel())


def apply_mapping(mapping: RunoffMapping, grid: torch.Tensor, out: Optional[torch.Tensor] = None,
                  dtype: Optional[torch.dtype] = None, unit_factor: float = 1.0,
                  missing_value: Optional[float] = None, clamp_negative: bool = False,
                  status: Optional[torch.Tensor] = None, stream: Optional[torch.cuda.Stream] = None
                  ) -> torch.Tensor:
    """Map a device chunk of gridded runoff onto the mapping's catchments.

    grid: [T, ny, nx] or [T, ny*nx] -> out [T, rows];
          [T, M, ny, nx] or [T, M, ny*nx] -> out [T, rows, M] (member innermost,
          the layout `set_inputs` takes for an ensemble).
    missing_value: grid entries that are NaN or equal to it (in the grid's
    dtype) are left out of the sum; clamp_negative sets negative sums to 0."""
    if grid.device.type != "cuda":
        raise ValueError("shard_forcing runs on the GPU: move the chunk to the device first")
    if grid.dtype not in _DTYPE_CODE:
        raise TypeError(f"grid dtype {grid.dtype} (float32 / float64 only)")
    G = mapping.num_cols
    if grid.dim() in (3, 4) and grid.shape[-1] != G and grid.shape[-2] * grid.shape[-1] == G:
        grid = grid.reshape(*grid.shape[:-2], G)        # [..., ny, nx] -> [..., ny * nx]
    if grid.dim() not in (2, 3) or grid.shape[-1] != G:
        raise ValueError(f"grid shape {tuple(grid.shape)} does not match a {G}-cell runoff grid")
    grid = grid.contiguous()
    T = int(grid.shape[0])
    M = int(grid.shape[1]) if grid.dim() == 3 else 1
    R = mapping.num_rows
    dtype = dtype or (out.dtype if out is not None else grid.dtype)
    if dtype not in _DTYPE_CODE:
        raise TypeError(f"output dtype {dtype} (float32 / float64 only)")
    shape = (T, R, M) if grid.dim() == 3 else (T, R)
    if out is None:
        out = torch.empty(shape, dtype=dtype, device=grid.device)
    elif tuple(out.shape) != shape or out.dtype != dtype or not out.is_contiguous() or out.device != grid.device:
        raise ValueError(f"out must be a contiguous {dtype} tensor of shape {shape} on {grid.device}")
    flags = (SKIP_MISSING if missing_value is not None else 0) | (CLAMP_NEGATIVE if clamp_negative else 0)
    h = _bind(_lib.lib())
    s = (stream or torch.cuda.current_stream(grid.device)).cuda_stream
    m = mapping._c()
    _lib.check(h.cmf_forcing_apply(
        ctypes.byref(m), s, grid.data_ptr(), _DTYPE_CODE[grid.dtype], T, M,
        M * G, G, out.data_ptr(), _DTYPE_CODE[dtype], R * M, 1, M,
        float(unit_factor), float("nan") if missing_value is None else float(missing_value),
        flags, status.data_ptr() if status is not None else None), "forcing_apply")
    return out


def shard_forcing(runoff_chunk: torch.Tensor, local_mapping: RunoffMapping, **kw) -> torch.Tensor:
    """hydroforge `dataset.shard_forcing` (scripts/run_daily_bin.py:116-119):
    [T, grid] on the device -> [T, catchments] in the mapping's row order."""
    return apply_mapping(local_mapping, runoff_chunk, **kw)


class MappedForcing:
    """Mixin giving a runoff dataset the two calls the reference's run scripts
    make on it (`build_local_mapping`, `shard_forcing`) backed by the GPU map.
    `unit_factor` (class or instance attribute, default 1) divides the mapped
    sum (as a multiplication by its reciprocal), as the reference datasets'
    `unit_factor` converts raw runoff units."""
    unit_factor: float = 1.0
    missing_value: Optional[float] = None
    clamp_negative: bool = False

    def build_local_mapping(self, mapping_file, desired_catchment_ids, device="cuda",
                            allow_missing: bool = False) -> RunoffMapping:
        return build_local_mapping(mapping_file, desired_catchment_ids, device, allow_missing)

    def shard_forcing(self, runoff_chunk: torch.Tensor, local_mapping: RunoffMapping,
                      dtype: Optional[torch.dtype] = None) -> torch.Tensor:
        return apply_mapping(local_mapping, runoff_chunk, dtype=dtype, unit_factor=self.unit_factor,
                             missing_value=self.missing_value, clamp_negative=self.clamp_negative)
