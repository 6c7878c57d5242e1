"""Edge cases of the routing path on the GPU, through the C ABI, against the
reference's own CUDA kernels (oracle/_ref, bit-exact):

* networks of 1 and 2 catchments and of sizes one past a CTA tile (33, 65, 257),
  at CTA sizes of 32, 64 and 256: the last, partial tile of every grid and the
  upstream range of the last cell;
* a dry start (zero river and flood storage and depth, water only in the dam
  cells the reservoir module fills) with and without runoff: the zero-depth
  guards of the momentum and stage equations;
* member counts that are not a power of two with member tiles that equal the
  member count or divide it (batched runs against one member per thread).
"""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn
from oracle import ref_cuda as RC

import parity as P

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not RC.available(), reason="oracle/_ref not built")


def _network(n: int, seed: int = 5) -> syn.Network:
    """Full physics where the size allows it (levees, paths, reservoirs)."""
    return syn.generate(syn.NetworkSpec(n, seed=seed, bifurcation_paths=n // 20,
                                        levee_fraction=0.25 if n >= 33 else 0.0,
                                        reservoirs=n // 100))


def _interval_vs_reference(net, orc, runoff, **model_kw):
    ref = P.ref_cuda_from_oracle(net, orc)
    model = P.model_for(net, **model_kw)
    P.load_oracle_state(model, orc)
    ref.set_runoff(runoff)
    model.set_inputs(torch.as_tensor(runoff[model.order]).cuda())
    n = ref.step_advance(86400.0)
    model.step_advance()
    torch.cuda.synchronize()
    assert int(model.sub_step_counts()[0].item()) == n
    P.assert_bit_exact(model, ref.state(), diag=True)
    model.check_status()
    return model


@needs_ref
@pytest.mark.parametrize("block", [32, 64, 256])
@pytest.mark.parametrize("n", [1, 2, 33, 65, 257])
def test_small_and_ragged_networks_bit_exact(n, block, device):
    net = _network(n)
    orc = P.oracle_for(net)
    P.spin_up(net, orc, days=1)
    _interval_vs_reference(net, orc, syn.daily_runoff(net, 3), BLOCK_SIZE=block)


@needs_ref
@pytest.mark.parametrize("runoff_scale", [0.0, 1.0])
def test_dry_start_bit_exact(runoff_scale, device):
    net = P.make_network("full", n=3000, seed=13)
    for k in ("river_storage", "flood_storage", "river_depth"):
        net.fields[k] = np.zeros_like(net.fields[k])
    orc = P.oracle_for(net)
    st = orc.state()
    # the reservoir module fills the dam cells (initialize_dam_storage), so
    # only those hold water at the start
    before = sum(float(np.sum(st[k])) for k in P.CELL_STO)
    runoff = (syn.daily_runoff(net, 0) * runoff_scale).astype(np.float32)
    model = _interval_vs_reference(net, orc, runoff)
    for k, v in model.state_tensors().items():
        assert torch.isfinite(v).all(), k
    after = sum(float(getattr(model.base, k).sum().item()) for k in P.CELL_STO)
    if runoff_scale == 0.0:
        assert after <= before * (1.0 + 1e-12)      # no source: water only leaves at mouths
    else:
        assert after > before


@pytest.mark.parametrize("members,width", [(3, 3), (6, 2), (6, 3), (6, 6)])
def test_member_tiles_of_odd_member_counts(members, width, device):
    net = syn.generate(syn.NetworkSpec(5_000, seed=17, bifurcation_paths=60, levee_fraction=0.2,
                                       reservoirs=5))
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=17)
    per = {"river_manning": (net.fields["river_manning"][:, None] * mfac).astype(np.float32)}
    kw = dict(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
              num_members=members, batched_fields=per, BLOCK_SIZE=64)
    ref, tiled = CaMaFlood(**kw), CaMaFlood(**kw)
    tiled.set_member_tile(width)
    order = ref.order
    for day in range(2):
        rm = torch.as_tensor((syn.daily_runoff(net, day)[:, None] * rfac).astype(np.float32)[order])
        for m in (ref, tiled):
            m.set_inputs(rm.to(device))
            m.step_advance()
    torch.cuda.synchronize()
    a, b = ref.state_tensors(), tiled.state_tensors()
    for k in a:
        np.testing.assert_array_equal(b[k].cpu().numpy(), a[k].cpu().numpy(), err_msg=k)
    tiled.check_status()
