"""Basin-sharded routing across ranks (one process per GPU).

Basins do not exchange water, so the network shards by basin with no data
exchange on the routing path.  The pieces:

* `basin_groups`   connected components of the river tree plus bifurcation
                   paths (a path joins its two basins), optionally merged by a
                   given `catchment_basin_id`; the reference shards by that
                   group field (cmfgpu/models/cama_flood_model.py:58-59) after
                   merging bifurcation-connected basins
                   (cmfgpu/params/utils.py:380-481);
* `lpt_assign`     Longest-Processing-Time assignment of groups to ranks by
                   cell count, the schedule the reference reports
                   (cmfgpu/params/merit_map.py:659-685): largest group first,
                   onto the least-loaded rank (lowest rank on ties);
* `shard_fields`   the input fields of one rank's catchments, paths, levees
                   and reservoirs, in input order;
* `ShardedRouting` one rank's model.  With `global_dt` (the reference's
                   behaviour) the CFL sub-step count is all-reduced with MAX
                   across ranks every interval
                   (cmfgpu/models/cama_flood_model.py:119-120), so every
                   basin advances with one dt.  Without it every rank keeps
                   its own dt and no collective runs.

The engine a rank drives is a `CaMaFlood` on its GPU by default; `engine`
takes any factory of an object with the same small protocol (`set_inputs`,
`local_sub_steps`, `advance`, `state`), which the CPU tests use.
"""
from __future__ import annotations

import heapq
from typing import Callable, Mapping, Optional

import numpy as np
import torch
import torch.distributed as dist

MODULE_FIELDS = {
    "bifurcation_catchment_id": ("bifurcation_catchment_id", "bifurcation_downstream_id",
                                 "bifurcation_path_id", "bifurcation_manning",
                                 "bifurcation_width", "bifurcation_length",
                                 "bifurcation_elevation", "bifurcation_outflow",
                                 "bifurcation_cross_section_depth"),
    "levee_catchment_id": ("levee_catchment_id", "levee_id", "levee_crown_height",
                           "levee_fraction"),
    "reservoir_catchment_id": ("reservoir_catchment_id", "reservoir_id", "reservoir_capacity",
                               "reservoir_area", "conservation_volume", "emergency_volume",
                               "normal_outflow", "flood_control_outflow"),
}


def _roots(parent: np.ndarray) -> np.ndarray:
    """Root of every node of a forest given as a parent array (pointer jumping)."""
    p = parent.copy()
    while True:
        q = p[p]
        if np.array_equal(q, p):
            return p
        p = q


def _id_index(fields: Mapping[str, np.ndarray]):
    """ids -> input index (searchsorted over the sorted catchment ids)."""
    cid = np.asarray(fields["catchment_id"], dtype=np.int64)
    srt = np.argsort(cid, kind="stable")
    sc = cid[srt]

    def index(ids):
        ids = np.asarray(ids, dtype=np.int64)
        pos = np.searchsorted(sc, ids).clip(0, max(sc.size - 1, 0))
        if ids.size and not np.array_equal(sc[pos], ids):
            raise ValueError("an id does not name a catchment of the network")
        return srt[pos]

    return index


def downstream_index(fields: Mapping[str, np.ndarray]) -> np.ndarray:
    """Downstream index from catchment/downstream ids (self at mouths)."""
    cid = np.asarray(fields["catchment_id"], dtype=np.int64)
    did = np.asarray(fields["downstream_id"], dtype=np.int64)
    srt = np.argsort(cid, kind="stable")
    pos = np.searchsorted(cid[srt], did).clip(0, cid.size - 1)
    hit = cid[srt][pos] == did
    return np.where(hit, srt[pos], np.arange(cid.size)).astype(np.int64)


def basin_groups(fields: Mapping[str, np.ndarray], modules=(), use_basin_id: bool = False) -> np.ndarray:
    """Group label per catchment (input order): catchments that must share a
    rank.  The label is the smallest catchment index of the group."""
    dn = downstream_index(fields)
    n = dn.size
    root = _roots(dn)                       # the mouth each catchment drains to
    parent = np.arange(n, dtype=np.int64)   # union-find over the mouths

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    pairs = []
    if "bifurcation" in set(modules) and "bifurcation_catchment_id" in fields:
        index = _id_index(fields)
        pairs.append(np.stack([root[index(fields["bifurcation_catchment_id"])],
                               root[index(fields["bifurcation_downstream_id"])]], axis=1))
    if use_basin_id and "catchment_basin_id" in fields:
        bid = np.asarray(fields["catchment_basin_id"], dtype=np.int64)
        order = np.argsort(bid, kind="stable")
        same = bid[order][1:] == bid[order][:-1]
        pairs.append(np.stack([root[order][:-1][same], root[order][1:][same]], axis=1))
    for pr in pairs:
        for a, b in np.unique(pr, axis=0):
            ra, rb = find(int(a)), find(int(b))
            if ra != rb:
                parent[max(ra, rb)] = min(ra, rb)
    labmap = np.arange(n, dtype=np.int64)
    for m in np.unique(root):
        labmap[m] = find(int(m))
    lab = labmap[root]
    first = np.full(n, n, dtype=np.int64)
    np.minimum.at(first, lab, np.arange(n))
    return first[lab]


def lpt_assign(sizes: np.ndarray, world_size: int) -> tuple[np.ndarray, np.ndarray]:
    """(rank of every group, load of every rank): largest group first onto
    the least-loaded rank, the lowest rank on ties."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    heap = [(0, r) for r in range(world_size)]
    rank = np.empty(sizes.size, dtype=np.int64)
    for g in order:
        load, r = heapq.heappop(heap)
        rank[g] = r
        heapq.heappush(heap, (load + int(sizes[g]), r))
    loads = np.zeros(world_size, dtype=np.int64)
    np.add.at(loads, rank, sizes)
    return rank, loads


def partition(fields: Mapping[str, np.ndarray], modules, world_size: int,
              use_basin_id: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """(rank of every catchment, cells per rank)."""
    groups = basin_groups(fields, modules, use_basin_id)
    _, inv, sizes = np.unique(groups, return_inverse=True, return_counts=True)
    grank, loads = lpt_assign(sizes, world_size)
    return grank[inv], loads


def shard_fields(fields: Mapping[str, np.ndarray], cell_rank: np.ndarray, rank: int) -> dict:
    """The input fields of the catchments of `rank` (input order kept), with
    the bifurcation paths, levees and reservoirs whose catchments it owns."""
    n = np.asarray(fields["catchment_id"]).shape[0]
    mine = cell_rank == rank
    module_names = {k for names in MODULE_FIELDS.values() for k in names}
    out = {}
    for k, v in fields.items():
        a = np.asarray(v)
        if k not in module_names and a.ndim >= 1 and a.shape[0] == n:
            out[k] = a[mine]
    index = _id_index(fields)
    for key, names in MODULE_FIELDS.items():
        if key not in fields:
            continue
        keep = mine[index(fields[key])]
        if key == "bifurcation_catchment_id":
            # both ends of a path share a group, hence a rank
            assert np.array_equal(keep, mine[index(fields["bifurcation_downstream_id"])])
        for k in names:
            if k in fields:
                out[k] = np.asarray(fields[k])[keep]
    return out


class ShardedRouting:
    """One rank of a basin-sharded model.

    fields / modules    the whole network (input order), identical on every rank
    rank, world_size    this process's place; `group` the process group
    global_dt           all-reduce the CFL count (MAX) every interval
    engine              factory (shard fields, modules) -> engine; default a
                        `CaMaFlood` on `device` built with `model_kwargs`
    """

    def __init__(self, fields: Mapping[str, np.ndarray], modules, rank: int, world_size: int,
                 device=None, group=None, global_dt: bool = True, use_basin_id: bool = False,
                 engine: Optional[Callable] = None, **model_kwargs):
        self.rank, self.world_size, self.group = int(rank), int(world_size), group
        self.global_dt = bool(global_dt)
        self.cell_rank, self.loads = partition(fields, modules, world_size, use_basin_id)
        self.local_input = np.flatnonzero(self.cell_rank == self.rank)   # global input indices
        local = shard_fields(fields, self.cell_rank, self.rank)
        if engine is None:
            from .model import CaMaFlood
            model = CaMaFlood(device=device, input_proxy=local, opened_modules=modules,
                              **model_kwargs)
            self.engine = ModelEngine(model)
        else:
            self.engine = engine(local, modules)
        nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"
        cdev = (torch.device(device) if device is not None else torch.device("cuda")) if nccl \
            else torch.device("cpu")
        self._count = torch.zeros(1, dtype=torch.int64, device=cdev)

    @property
    def imbalance(self) -> float:
        """Largest relative deviation of a rank's cell count from the mean."""
        avg = self.loads.sum() / max(1, self.world_size)
        return float(np.max(np.abs(self.loads - avg)) / avg) if avg > 0 else 0.0

    def set_inputs(self, runoff_global: np.ndarray) -> None:
        """Runoff of the whole network (input order); each rank takes its part."""
        self.engine.set_inputs(np.asarray(runoff_global)[self.local_input])

    def sub_steps(self) -> int:
        """This interval's sub-step count: the local CFL count, or its maximum
        over ranks with `global_dt`."""
        n = int(self.engine.local_sub_steps())
        if self.global_dt and self.world_size > 1:
            self._count.fill_(n)
            dist.all_reduce(self._count, op=dist.ReduceOp.MAX, group=self.group)
            n = int(self._count.item())
        return n

    def step_advance(self) -> int:
        n = self.sub_steps()
        self.engine.advance(n)
        return n

    def gather_state(self, names) -> Optional[dict]:
        """Rank 0 receives the listed state fields of every rank reassembled in
        global input order; the other ranks get None."""
        local = self.engine.state()
        out = {} if self.rank == 0 else None
        for name in names:
            piece = np.ascontiguousarray(local[name])
            if self.world_size > 1:
                parts = [None] * self.world_size if self.rank == 0 else None
                dist.gather_object(piece, parts, dst=0, group=self.group)
            else:
                parts = [piece]
            if self.rank == 0:
                full = np.empty((self.cell_rank.size,) + parts[0].shape[1:], dtype=parts[0].dtype)
                for r in range(self.world_size):
                    full[self.cell_rank == r] = parts[r]
                out[name] = full
        return out


class ModelEngine:
    """The engine protocol over a CaMaFlood model (local input order in/out)."""

    def __init__(self, model):
        self.model = model
        self.order = model.order

    def set_inputs(self, runoff_local: np.ndarray) -> None:
        x = torch.as_tensor(np.ascontiguousarray(np.asarray(runoff_local)[self.order]))
        self.model.set_inputs(x.to(self.model.device))

    def local_sub_steps(self) -> int:
        self.model.compute_adaptive_time_step()
        return int(self.model.sub_step_counts()[0].item())

    def advance(self, n: int) -> None:
        self.model.step_advance(num_sub_steps=n)

    def state(self) -> dict:
        """Catchment-indexed state fields in local input order, plus the path
        fields (bifurcation order is kept as given)."""
        inv = self.model.inverse_order
        n = self.model.num_catchments
        out = {}
        for k, v in self.model.state_tensors().items():
            a = v.detach().cpu().numpy()
            cell = k not in ("bifurcation_outflow", "bifurcation_cross_section_depth")
            out[k] = a[inv] if cell and a.shape[0] == n else a
        return out
