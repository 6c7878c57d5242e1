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
