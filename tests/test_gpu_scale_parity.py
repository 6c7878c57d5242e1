"""Parity at the sizes of the benchmark workloads, against the reference's own
CUDA kernels (oracle/_ref: the cmfgpu/phys/cuda sources compiled unmodified for
sm_100a, stepped in the phase order of cmfgpu/models/cama_flood_model.py:134-162).

* plain_60k: 60,000 catchments, the full 30-day window with the 3600 s dt cap.
  The reference has no cap, so its arm runs the capped count max(n, 24) as a
  fixed sub-step count (86400 s / 3600 s = 24); the product applies the cap in
  its CFL kernel.  Both must agree on the count every day and end bit-exact.
  The error of the mixed-precision result against an fp64 oracle run of the
  same 30 days (same counts) is printed and held under bounds.
* full_250k: the first 10 simulated days of the 365-day full-physics run
  (8,000 bifurcation paths, levees on 20 % of cells, 500 reservoirs).
* full_6m: two simulated days of hourly intervals of the 6M-catchment
  full-physics roofline case (200,000 paths, ~977,000 levees, 7,000
  reservoirs), so the compared interval starts from a flooded state.

Every state field must be bit-identical.  The fp64 inflow diagnostics are
compared exactly too: a sum of a cell's few fp32 upstream fluxes is exact in
fp64, so the reference's fp64 atomic scatter and the product's ordered gather
agree although they add in different orders.
"""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn
from oracle import oracle as O, ref_cuda as RC

import parity as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RC.available(), reason="oracle/_ref not built")]


def _pair(name, **model_kw):
    cfg = syn.CONFIGS[name]
    net = syn.generate(cfg["spec"])
    mods = net.opened_modules
    model = CaMaFlood(device="cuda:0", input_proxy=net.fields, opened_modules=mods,
                      step_duration=cfg["interval"], **model_kw)
    ref = RC.RefCuda(O.reference_fields(net.fields, mods), mods)
    return cfg, net, model, ref


def _mismatches(model, ref) -> dict:
    st = ref.state()
    order = model.order
    out = {}
    for k, v in model.state_tensors().items():
        a = v.cpu().numpy()
        b = st[k] if a.ndim == 2 else st[k][order]
        out[k] = int(np.count_nonzero(a != b))
    for k in ("river_inflow", "flood_inflow"):
        out[k] = int(np.count_nonzero(getattr(model.base, k).cpu().numpy() != st[k][order]))
    return out


def _hourly(net, cfg, interval_index):
    d, h = divmod(interval_index, 24)
    prof = syn.diurnal_profile(d, seed=net.spec.seed, hours=24)
    return syn.daily_runoff(net, d) * prof[h]


def test_plain_60k_30_days_capped_dt(device):
    cfg, net, model, ref = _pair("plain_60k", max_sub_step_seconds=3600.0)
    orc = P.oracle_for(net, "float64")
    cap = int(round(86400.0 / cfg["max_sub_step_seconds"]))
    counts = []
    for d in range(cfg["days"]):
        r = syn.daily_runoff(net, d)
        ref.set_runoff(r)
        model.set_inputs(torch.as_tensor(r[model.order]).to(device))
        n = max(ref.adaptive_sub_steps(86400.0), cap)
        ref.step_advance(86400.0, adaptive=False, fixed_n=n)
        model.step_advance()
        n_model = int(model.sub_step_counts()[0].item())
        assert n_model == n, (d, n_model, n)
        orc.set_runoff(r)
        orc.step_advance(86400.0, adaptive=False, fixed_n=n)
        counts.append(n)
    torch.cuda.synchronize()
    mism = _mismatches(model, ref)
    assert not any(mism.values()), mism
    # error of the (bit-identical) mixed-precision result against fp64
    order = model.order
    print(f"\nplain_60k, 30 days, {sum(counts)} sub-steps: mixed precision vs fp64 oracle "
          "(max rel, p99 rel)")
    for k in P.CELL_REAL + P.CELL_STO:
        a = getattr(model.base, k).cpu().numpy().astype(np.float64)
        b = orc.a[k][order]
        floor = max(float(np.mean(np.abs(b))) * 1e-3, 1e-30)
        rel = np.abs(a - b) / (np.abs(b) + floor)
        mx, p99 = float(rel.max()) if rel.size else 0.0, float(np.quantile(rel, 0.99))
        print(f"  {k:36s} {mx:9.2e} {p99:9.2e}")
        if k in ("river_storage", "flood_storage", "river_depth", "river_outflow"):
            assert p99 < 1e-3, (k, mx, p99)


def test_full_250k_first_10_days(device):
    cfg, net, model, ref = _pair("full_250k")
    for d in range(10):
        r = syn.daily_runoff(net, d)
        ref.set_runoff(r)
        model.set_inputs(torch.as_tensor(r[model.order]).to(device))
        n = ref.step_advance(86400.0)
        model.step_advance()
        assert int(model.sub_step_counts()[0].item()) == n, d
    torch.cuda.synchronize()
    mism = _mismatches(model, ref)
    assert not any(mism.values()), mism


def test_full_6m_hourly_two_days(device):
    cfg, net, model, ref = _pair("full_6m")
    runoff_dev = ref.t["runoff"]
    for k in range(48):
        r = _hourly(net, cfg, k)
        runoff_dev.copy_(torch.as_tensor(r))
        model.set_inputs(torch.as_tensor(r[model.order]).to(device))
        n = ref.step_advance(3600.0)
        model.step_advance()
        assert int(model.sub_step_counts()[0].item()) == n, k
    torch.cuda.synchronize()
    mism = _mismatches(model, ref)
    flooded = float((model.base.flood_storage > 0).double().mean().item())
    print(f"\nfull_6m after 48 hourly intervals: flooded cell fraction {flooded:.3f}, "
          f"mismatching elements {mism}")
    assert not any(mism.values()), mism
