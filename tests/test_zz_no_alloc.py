"""cmf_substep_noalloc: the sub-step for callers that cannot allocate device
memory (inside a stream capture, or under a host that owns every buffer).

Through the C ABI it must produce exactly what the plan-based entry points
(cmf_phase_momentum + cmf_phase_stage) produce on an identical model, on two
calls in a row -- the second call runs on the static scratch the first call
left behind.  This file is collected last so that a failure here comes after
every other test has run."""
import ctypes

import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, _lib, synthetic as syn

pytestmark = pytest.mark.gpu


def _model(net):
    return CaMaFlood(device="cuda:0", input_proxy=net.fields, opened_modules=net.opened_modules)


@pytest.mark.parametrize("spec", [
    syn.NetworkSpec(5000, seed=31),
    syn.NetworkSpec(5000, seed=32, bifurcation_paths=200, levee_fraction=0.2, reservoirs=20),
])
def test_noalloc_substep_matches_plan_entry_points(spec, device):
    net = syn.generate(spec)
    ref = _model(net)          # plan-based entry points
    dut = _model(net)          # allocation-free entry point
    runoff = torch.as_tensor(syn.daily_runoff(net, 0)[ref.order]).cuda()
    ref.set_inputs(runoff)
    dut.set_inputs(runoff)
    ref.compute_adaptive_time_step()
    dut.base.time_step.copy_(ref.base.time_step)
    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        ref.compute_momentum(diag=True)
        ref.compute_stage(diag=True)
        rc = lib.cmf_substep_noalloc(ctypes.byref(dut._view_struct), stream, 1)
        assert rc == _lib.CMF_OK, lib.cmf_status_string(rc)
    torch.cuda.synchronize()
    a, b = ref.state_tensors(), dut.state_tensors()
    for k in a:
        np.testing.assert_array_equal(b[k].cpu().numpy(), a[k].cpu().numpy(), err_msg=k)
    for k in ("river_inflow", "flood_inflow"):
        np.testing.assert_array_equal(getattr(dut.base, k).cpu().numpy(),
                                      getattr(ref.base, k).cpu().numpy(), err_msg=k)


def _two_calls_each_way(ref, dut, net, budget=False):
    runoff = torch.as_tensor(syn.daily_runoff(net, 0)[ref.order]).cuda().to(ref.real_torch)
    ref.set_inputs(runoff)
    dut.set_inputs(runoff)
    ref.compute_adaptive_time_step()
    dut.base.time_step.copy_(ref.base.time_step)
    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        ref.compute_momentum(diag=True)
        ref.compute_stage(diag=True)
        if budget:
            ref.flush_budget()       # the allocation-free entry flushes every call
        rc = lib.cmf_substep_noalloc(ctypes.byref(dut._view_struct), stream, 1)
        assert rc == _lib.CMF_OK, lib.cmf_status_string(rc)
    torch.cuda.synchronize()
    a, b = ref.state_tensors(), dut.state_tensors()
    for k in a:
        np.testing.assert_array_equal(b[k].cpu().numpy(), a[k].cpu().numpy(), err_msg=k)


def test_noalloc_fp64_with_budget(device):
    """fp64 view with the water budget: state and budget equal the plan path's
    after two calls (the budget partials in the static array are cleared and
    flushed by every call)."""
    net = syn.generate(syn.NetworkSpec(4000, seed=34, bifurcation_paths=100, levee_fraction=0.2,
                                       reservoirs=10))
    kw = dict(device="cuda:0", input_proxy=net.fields, opened_modules=net.opened_modules,
              precision="float64", budget=True)
    ref, dut = CaMaFlood(**kw), CaMaFlood(**kw)
    _two_calls_each_way(ref, dut, net, budget=True)
    np.testing.assert_array_equal(dut.log.budget.cpu().numpy(), ref.log.budget.cpu().numpy())


def test_noalloc_near_capacity_small_ctas(device):
    """65,000 catchments with 32-thread CTAs: the largest per-CTA budget
    partial area the array must hold."""
    net = syn.generate(syn.NetworkSpec(65000, seed=35))
    kw = dict(device="cuda:0", input_proxy=net.fields, opened_modules=net.opened_modules,
              BLOCK_SIZE=32, budget=True)
    ref, dut = CaMaFlood(**kw), CaMaFlood(**kw)
    _two_calls_each_way(ref, dut, net, budget=True)
    np.testing.assert_array_equal(dut.log.budget.cpu().numpy(), ref.log.budget.cpu().numpy())


def test_noalloc_rejects_views_beyond_its_capacity(device):
    net = syn.generate(syn.NetworkSpec(70000, seed=33))
    m = _model(net)
    rc = _lib.lib().cmf_substep_noalloc(ctypes.byref(m._view_struct),
                                        torch.cuda.current_stream().cuda_stream, 0)
    assert rc == _lib.CMF_ERR_ARG
