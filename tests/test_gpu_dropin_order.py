"""The reference-facing adapter (cmfb200.registry.B200Backend) takes runoff in
the REFERENCE model's catchment order and hands state back in that order,
while the library routes in its own breadth-first order.  Feeding
reference-order runoff through the adapter must give, bit for bit, the state
of a model fed model-order runoff, and `set_inputs(order="input")` must equal
a host-side permutation."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn
from cmfb200.registry import B200Backend

pytestmark = pytest.mark.gpu


def test_reference_order_runoff_through_the_adapter(device):
    net = syn.generate(syn.NetworkSpec(5000, seed=41, bifurcation_paths=150, levee_fraction=0.2,
                                       reservoirs=15))
    mods = net.opened_modules
    direct = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods)
    adapter = B200Backend(net.fields, mods, device=device)
    np.testing.assert_array_equal(adapter.catchment_id, net.fields["catchment_id"])
    for d in range(2):
        r = syn.daily_runoff(net, d)                       # generator (= reference) order
        direct.set_inputs(torch.as_tensor(r[direct.order]).to(device))
        adapter.set_inputs(torch.as_tensor(r).to(device))
        direct.step_advance()
        adapter.step_advance()
    torch.cuda.synchronize()
    got = adapter.state()
    for k, v in direct.state_tensors().items():
        want = v.cpu().numpy()
        if not k.startswith("bifurcation_"):
            want = want[direct.inverse_order]
        np.testing.assert_array_equal(got[k].cpu().numpy(), want, err_msg=k)
    # write_back into reference-order tensors
    tgt = {"river_storage": torch.zeros(net.num_catchments, dtype=torch.float64, device=device)}
    adapter.write_back(tgt)
    np.testing.assert_array_equal(tgt["river_storage"].cpu().numpy(),
                                  got["river_storage"].cpu().numpy())
    adapter.close()
    direct.close()


def test_input_order_equals_host_permutation_for_members(device):
    net = syn.generate_basins(5, 3000, seed=2)
    m = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=["base", "adaptive_time"],
                  num_members=3)
    r = np.random.default_rng(0).random((net.num_catchments, 3)).astype(np.float32)
    m.set_inputs(torch.as_tensor(r).to(device), order="input")
    np.testing.assert_array_equal(m.base.runoff.cpu().numpy(), r[m.order])
    with pytest.raises(ValueError):
        m.set_inputs(torch.as_tensor(r).to(device), order="bfs")
    m.close()


def test_model_from_parameter_file_equals_model_from_fields(device, tmp_path):
    """A model built from a NetCDF-classic parameter file (reference axis
    names) routes exactly like one built from the in-memory fields."""
    from cmfb200.model import InputProxy
    from cmfb200 import params as PR
    net = syn.generate(syn.NetworkSpec(4000, seed=43, bifurcation_paths=100, levee_fraction=0.2,
                                       reservoirs=10))
    path = tmp_path / "parameters.nc"
    PR.write_parameters(path, net.fields)
    a = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules)
    b = CaMaFlood(device=device, input_proxy=InputProxy.from_nc(str(path)),
                  opened_modules=net.opened_modules)
    r = syn.daily_runoff(net, 0)
    for m in (a, b):
        m.set_inputs(torch.as_tensor(r).to(device), order="input")
        m.step_advance()
    torch.cuda.synchronize()
    for k, v in a.state_tensors().items():
        np.testing.assert_array_equal(b.state_tensors()[k].cpu().numpy(), v.cpu().numpy(), err_msg=k)
    a.close()
    b.close()
