"""Block-size autotuner (cmfb200.autotune): it leaves the state untouched,
keeps one of the candidates, caches its choice, and the tuned plan routes
exactly as a plan built with that block size directly (the kernels are
per-cell, so the CTA size changes no result)."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn

pytestmark = pytest.mark.gpu


def test_autotune_keeps_state_and_results(device, tmp_path):
    net = syn.generate(syn.NetworkSpec(20_000, seed=43, bifurcation_paths=200,
                                       levee_fraction=0.2, reservoirs=20))
    mods = net.opened_modules
    model = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods)
    r0 = torch.as_tensor(syn.daily_runoff(net, 0)[model.order]).to(device)
    model.set_inputs(r0)
    model.step_advance()
    before = {k: v.clone() for k, v in model.state_tensors().items()}
    cache = str(tmp_path / "tune.json")
    res = model.autotune_block_size(candidates=(64, 256), sub_steps=4, cache_path=cache)
    assert res["block_size"] in (64, 256) and not res["cached"]
    assert model.block_size == res["block_size"]
    for k, v in model.state_tensors().items():
        assert torch.equal(v, before[k]), k
    again = model.autotune_block_size(candidates=(64, 256), cache_path=cache)
    assert again["cached"] and again["block_size"] == res["block_size"]

    ref = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods,
                    BLOCK_SIZE=256 if res["block_size"] == 64 else 64)
    for k, v in ref.state_tensors().items():
        v.copy_(before[k])
    r1 = torch.as_tensor(syn.daily_runoff(net, 1)[model.order]).to(device)
    for m in (model, ref):
        m.set_inputs(r1)
        m.step_advance()
    for k, v in model.state_tensors().items():
        np.testing.assert_array_equal(v.cpu().numpy(), ref.state_tensors()[k].cpu().numpy(), err_msg=k)
