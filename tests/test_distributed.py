"""Basin sharding across ranks (cmfb200.distributed) on CPU.

* The partition: groups are closed under the river tree and bifurcation
  paths, every catchment/path/levee/reservoir lands on exactly one rank, and
  the LPT loads equal the greedy schedule the reference reports.
* The multi-rank step: two gloo ranks each route their shard with the fp64 C
  oracle as the engine.  With the global dt (CFL count all-reduced with MAX,
  the reference's behaviour) the gathered state equals one oracle run over
  the whole network bit for bit, because basins exchange no water.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cmfb200 import distributed as D, synthetic as syn
from oracle import oracle as O

STATE = ("river_storage", "flood_storage", "river_outflow", "flood_outflow", "river_depth",
         "flood_depth", "flood_fraction")
OUTER = 86400.0


class OracleEngine:
    """The engine protocol over the fp64 C oracle (test infrastructure).  One
    thread: the oracle scatters inflow with atomics as the reference does, so
    only a sequential run fixes the summation order."""

    def __init__(self, fields, modules):
        O.set_threads(1)
        f = O.reference_fields(fields, modules, "float64")
        self.orc = O.Oracle(f, modules, "float64")

    def set_inputs(self, runoff):
        self.orc.set_runoff(runoff)

    def local_sub_steps(self):
        return self.orc.adaptive_sub_steps(OUTER)

    def advance(self, n):
        self.orc.step_advance(OUTER, adaptive=False, fixed_n=n)

    def state(self):
        st = self.orc.state()
        return {k: st[k] for k in STATE}


def _network(case="plain"):
    extra = dict(levee_fraction=0.0) if case == "plain" else dict(
        levee_fraction=0.2, reservoirs=12, bifurcation_paths=20)
    return syn.generate(syn.NetworkSpec(6000, seed=31, **extra))


def test_partition_is_closed_and_complete():
    net = _network("full")
    f, mods = net.fields, net.opened_modules
    groups = D.basin_groups(f, mods)
    dn = D.downstream_index(f)
    assert np.array_equal(groups, groups[dn])                      # river edges inside groups
    idx = D._id_index(f)
    a, b = idx(f["bifurcation_catchment_id"]), idx(f["bifurcation_downstream_id"])
    assert np.array_equal(groups[a], groups[b])                    # paths inside groups
    for world in (1, 2, 3, 4):
        cell_rank, loads = D.partition(f, mods, world)
        assert loads.sum() == dn.size
        assert np.array_equal(cell_rank, cell_rank[dn])            # no river edge crosses ranks
        shards = [D.shard_fields(f, cell_rank, r) for r in range(world)]
        ids = np.concatenate([s["catchment_id"] for s in shards])
        assert np.array_equal(np.sort(ids), np.sort(f["catchment_id"]))
        for key in ("levee_catchment_id", "reservoir_catchment_id", "bifurcation_catchment_id"):
            assert sum(s[key].size for s in shards) == f[key].size


def _greedy_loads(sizes, bins):
    """Each size, largest first, onto the least-loaded bin (first on ties)."""
    loads = [0] * bins
    for s in sorted(sizes, reverse=True):
        j = loads.index(min(loads))
        loads[j] += int(s)
    return loads


def test_lpt_loads_match_greedy_schedule():
    rng = np.random.default_rng(0)
    for bins in (1, 2, 3, 8):
        sizes = rng.integers(1, 10_000, size=200)
        rank, loads = D.lpt_assign(sizes, bins)
        assert list(loads) == _greedy_loads(sizes, bins)
        assert np.array_equal(np.bincount(rank, weights=sizes, minlength=bins).astype(np.int64), loads)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, days, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = _network(case)
        sr = D.ShardedRouting(net.fields, net.opened_modules, rank, world, global_dt=True,
                              engine=OracleEngine)
        counts = []
        for d in range(days):
            sr.set_inputs(syn.daily_runoff(net, d))
            counts.append(sr.step_advance())
        st = sr.gather_state(STATE)
        if rank == 0:
            np.savez(out_path, counts=np.array(counts), **st)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["plain", "full"])
def test_two_ranks_equal_one_process(case, tmp_path):
    days, world = 3, 2
    out = str(tmp_path / "ranks.npz")
    mp.start_processes(_worker, args=(world, _free_port(), case, days, out), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(out)
    net = _network(case)
    eng = OracleEngine(net.fields, net.opened_modules)
    counts = []
    for d in range(days):
        eng.set_inputs(syn.daily_runoff(net, d))
        n = eng.local_sub_steps()
        eng.advance(n)
        counts.append(n)
    assert list(got["counts"]) == counts
    ref = eng.state()
    for k in STATE:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
