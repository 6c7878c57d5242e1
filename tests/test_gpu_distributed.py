"""The basin-sharded wrapper (cmfb200.distributed.ShardedRouting) driving
the CUDA model on one GPU: a single rank owns every basin, so it must equal a
plain CaMaFlood run of the same network bit for bit, with the sub-step count
taken through the wrapper's CFL path and passed back as a fixed count."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, distributed as D, synthetic as syn

pytestmark = pytest.mark.gpu

STATE = ("river_storage", "flood_storage", "river_outflow", "flood_outflow", "river_depth",
         "flood_depth", "flood_fraction", "protected_storage")


@pytest.mark.parametrize("case", ["plain", "full"])
def test_single_rank_equals_plain_model(case, device):
    extra = dict(levee_fraction=0.0) if case == "plain" else dict(
        levee_fraction=0.2, reservoirs=12, bifurcation_paths=40)
    net = syn.generate(syn.NetworkSpec(8000, seed=41, **extra))
    sr = D.ShardedRouting(net.fields, net.opened_modules, 0, 1, device=device)
    plain = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules)
    for d in range(3):
        r = syn.daily_runoff(net, d)
        sr.set_inputs(r)
        n = sr.step_advance()
        plain.set_inputs(torch.as_tensor(r[plain.order]).to(device))
        plain.step_advance()
        assert n == int(plain.sub_step_counts()[0].item())
    got = sr.gather_state(STATE)
    for k in STATE:
        ref = getattr(plain.base, k).cpu().numpy()[plain.inverse_order]
        np.testing.assert_array_equal(got[k], ref, err_msg=k)


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _network(case):
    extra = dict(levee_fraction=0.0) if case == "plain" else dict(
        levee_fraction=0.2, reservoirs=12, bifurcation_paths=20)
    return syn.generate(syn.NetworkSpec(8000, seed=31, **extra))


def _rank_worker(rank, world, port, case, days, out_path):
    import os
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = _network(case)
        sr = D.ShardedRouting(net.fields, net.opened_modules, rank, world, device="cuda:0",
                              global_dt=True)
        counts = []
        for d in range(days):
            sr.set_inputs(syn.daily_runoff(net, d))
            counts.append(sr.step_advance())
        st = sr.gather_state(STATE)
        if rank == 0:
            np.savez(out_path, counts=np.array(counts), loads=sr.loads, **st)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["plain", "full"])
def test_two_ranks_of_the_cuda_model_equal_one_model(case, device, tmp_path):
    """Two ranks, each a separate process driving the CUDA model on its own
    basins (both on this one GPU; their kernels never wait on each other),
    with the sub-step count all-reduced (MAX) over a gloo group on the host:
    the gathered state equals one whole-network model bit for bit."""
    import torch.multiprocessing as mp
    days, world = 3, 2
    out = str(tmp_path / "ranks.npz")
    mp.start_processes(_rank_worker, args=(world, _free_port(), case, days, out), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(out)
    assert (got["loads"] > 0).all()                       # both ranks own basins
    net = _network(case)
    plain = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules)
    counts = []
    for d in range(days):
        plain.set_inputs(torch.as_tensor(syn.daily_runoff(net, d)[plain.order]).to(device))
        plain.step_advance()
        counts.append(int(plain.sub_step_counts()[0].item()))
    assert list(got["counts"]) == counts
    for k in STATE:
        ref = getattr(plain.base, k).cpu().numpy()[plain.inverse_order]
        np.testing.assert_array_equal(got[k], ref, err_msg=k)
