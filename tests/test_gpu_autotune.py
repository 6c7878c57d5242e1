"""Block-size and member-tile autotuner (cmfb200.autotune): it leaves the
state untouched, keeps one of the candidates, caches its choice, and the tuned
plan routes exactly as a plan built with that block size directly (the kernels
are per-cell, so the CTA size and member tile change no result)."""
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


def test_autotune_member_tile(device, tmp_path):
    members = 4
    net = syn.generate_basins(30, 20_000, seed=5)
    rfac, mfac = syn.ensemble_factors(net.num_catchments, members, seed=5)
    manning = (net.fields["river_manning"][:, None] * mfac).astype(np.float32)
    kw = dict(device=device, input_proxy=net.fields, opened_modules=["base", "adaptive_time"],
              num_members=members, batched_fields={"river_manning": manning})
    model = CaMaFlood(**kw)
    order = model.order
    rm = torch.as_tensor((syn.daily_runoff(net, 0)[:, None] * rfac).astype(np.float32)[order]).to(device)
    model.set_inputs(rm)
    model.step_advance()
    before = {k: v.clone() for k, v in model.state_tensors().items()}
    cache = str(tmp_path / "tune.json")
    res = model.autotune_block_size(candidates=(128, 256), sub_steps=4, cache_path=cache,
                                    tile_candidates=(1, 2, 3, 4))
    assert set(res["ms_per_sub_step"]) == {f"{b}/{w}" for b in (128, 256) for w in (1, 2, 4)}
    assert (model.block_size, model.member_tile) == (res["block_size"], res["member_tile"])
    for k, v in model.state_tensors().items():
        assert torch.equal(v, before[k]), k
    again = model.autotune_block_size(candidates=(128, 256), cache_path=cache)
    assert again["cached"] and again["member_tile"] == res["member_tile"]
    ref = CaMaFlood(**kw)
    for k, v in ref.state_tensors().items():
        v.copy_(before[k])
    rm1 = torch.as_tensor((syn.daily_runoff(net, 1)[:, None] * rfac).astype(np.float32)[order]).to(device)
    for m in (model, ref):
        m.set_inputs(rm1)
        m.step_advance()
    for k, v in model.state_tensors().items():
        assert torch.equal(v, ref.state_tensors()[k]), k
