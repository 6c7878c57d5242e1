"""The CUDA product against golden fixtures made by the reference's own CUDA
kernels (tests/golden/make_ref_golden.py): one sub-step from a stored state,
bit-exact, and the same CFL sub-step count."""
from pathlib import Path

import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn

import golden_cases as G

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"


@pytest.mark.parametrize("case", list(G.CASES))
def test_product_matches_reference_golden(case, device):
    path = GOLD / f"ref_{case}.npz"
    if not path.exists():
        pytest.skip("fixture not generated")
    g = np.load(path)
    net = syn.generate(G.CASES[case])
    m = CaMaFlood(device="cuda:0", input_proxy=net.fields, opened_modules=net.opened_modules)
    order = m.order
    for k in G.state_fields(net.opened_modules):
        a = g["in_" + k]
        t = m.state_tensors()[k]
        t.copy_(torch.as_tensor(a if k.startswith("bifurcation") else a[order]))
    m.set_inputs(torch.as_tensor(syn.daily_runoff(net, 1)[order]).cuda())
    m.compute_adaptive_time_step()
    assert int(m.sub_step_counts()[0].item()) == int(g["n"])
    assert float(m.base.time_step[0].item()) == float(g["dt"])
    m.compute_momentum(diag=True)
    m.compute_stage(diag=True)
    torch.cuda.synchronize()
    for k in G.state_fields(net.opened_modules):
        ours = m.state_tensors()[k].cpu().numpy()
        ref = g["out_" + k] if k.startswith("bifurcation") else g["out_" + k][order]
        np.testing.assert_array_equal(ours, ref, err_msg=k)
    for k in ("river_inflow", "flood_inflow"):
        np.testing.assert_array_equal(getattr(m.base, k).cpu().numpy(), g["out_" + k][order], err_msg=k)
