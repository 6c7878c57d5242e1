"""The persistent interval kernel (cmf_plan_set_persistent): every sub-step of
an interval in one cooperative launch, the phases separated by grid-wide
barriers.  It calls the same per-element device functions as the four
sub-step kernels, so its state must equal the interval graph's bit for bit,
in every feature case, in fp32 and fp64, with the grid smaller than the work
(grid-stride loops) and larger CTAs; and it must refuse what it does not
support."""
import numpy as np
import pytest
import torch

from cmfb200 import synthetic as syn

import parity as P

pytestmark = pytest.mark.gpu


def _run(net, days, persistent, **kw):
    m = P.model_for(net, persistent=persistent, **kw)
    counts = []
    for d in range(days):
        m.set_inputs(torch.as_tensor(m.to_model_order(syn.daily_runoff(net, d))).cuda())
        m.step_advance()
        counts.append(int(m.sub_step_counts()[0].item()))
    torch.cuda.synchronize()
    m.check_status()
    state = {k: v.cpu().numpy().copy() for k, v in m.state_tensors().items()}
    return state, counts


def _assert_equal(a, b):
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("case", list(P.CASES))
def test_persistent_equals_graph(case, device):
    net = P.make_network(case)
    g, cg = _run(net, 2, False)
    p, cp = _run(net, 2, True)
    assert cg == cp
    _assert_equal(g, p)


def test_persistent_fp64_full_physics(device):
    net = P.make_network("full")
    g, cg = _run(net, 2, False, precision="float64")
    p, cp = _run(net, 2, True, precision="float64")
    assert cg == cp
    _assert_equal(g, p)


@pytest.mark.parametrize("block", [64, 256])
def test_persistent_grid_stride_on_a_large_network(block, device):
    """200k catchments: more work items than resident threads, so every block
    walks several cells per phase."""
    net = P.make_network("full", n=200000, seed=8)
    g, cg = _run(net, 1, False, BLOCK_SIZE=block)
    p, cp = _run(net, 1, True, BLOCK_SIZE=block)
    assert cg == cp
    _assert_equal(g, p)


def test_persistent_fixed_sub_steps_and_switching(device):
    """Fixed sub-step counts, and switching between graph and persistent
    intervals inside one run."""
    net = P.make_network("full", seed=4)
    ref = P.model_for(net)
    mix = P.model_for(net)
    for d in range(4):
        r = torch.as_tensor(ref.to_model_order(syn.daily_runoff(net, d))).cuda()
        mix.set_persistent(d % 2 == 0)
        for m in (ref, mix):
            m.set_inputs(r)
            m.step_advance(num_sub_steps=40 if d == 3 else None)
    torch.cuda.synchronize()
    mix.check_status()
    _assert_equal({k: v.cpu().numpy() for k, v in ref.state_tensors().items()},
                  {k: v.cpu().numpy() for k, v in mix.state_tensors().items()})


def test_persistent_refuses_what_it_does_not_run(device):
    net = P.make_network("plain", n=2000)
    with pytest.raises(ValueError):
        P.model_for(net, budget=True, persistent=True)
    with pytest.raises(ValueError):
        P.model_for(net, variables_to_save={"mean": ["total_outflow"]}, persistent=True)
    rf = np.ones((net.num_catchments, 2), dtype=np.float32)
    with pytest.raises(ValueError):
        P.model_for(net, num_members=2, batched_fields={"river_manning": rf}, persistent=True)


def test_barrier_wait_gives_up_and_reports(device):
    """The persistent kernel's barrier is bounded: a barrier that waits for
    one arrival more than the grid makes (a count nothing completes) gives up
    after its time limit, reports CMF_STATUS_SYNC_TIMEOUT and the abort word,
    and the kernel returns; the context stays usable."""
    import time
    from cmfb200 import _lib
    ctl = torch.zeros(16, dtype=torch.int32, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    t0 = time.perf_counter()
    rc = _lib.lib().cmf_probe_barrier_timeout(stream, ctl.data_ptr(), status.data_ptr(), 20000)
    assert rc == _lib.CMF_OK
    torch.cuda.synchronize(device)
    assert time.perf_counter() - t0 < 10.0
    assert int(status.item()) & _lib.STATUS_SYNC_TIMEOUT
    c = ctl.cpu().numpy()
    assert c[6] == 1                                    # abort word
    assert int(c[4]) + (int(c[5]) << 32) == 2           # both blocks arrived once
    x = torch.arange(100, device=device, dtype=torch.float32)
    assert float(x.sum().item()) == 4950.0
