"""Output statistics accumulated on the device (variables_to_save) against
(1) a replay through the per-phase entry points with torch fp64 arithmetic
    in the same operation order -- bit-exact,
(2) the CPU oracle stepped sub-step by sub-step with oracle.forcing.StatsReplay
    -- fp64 storage and fp64 fluxes, 1e-10 relative,
(3) single-member runs, member by member, for a batched ensemble whose
    members take different sub-step counts -- bit-exact."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn, _lib
from oracle import forcing as OF

import parity as P

pytestmark = pytest.mark.gpu

FLUX_DEPTH = {"mean": ["total_outflow", "river_outflow", "river_depth", "flood_fraction"],
              "max": ["total_outflow", "flood_depth"], "min": ["river_depth"],
              "last": ["river_depth", "flood_depth"]}
WITH_STORAGE = {"mean": ["total_outflow", "river_storage", "flood_storage", "protected_depth"],
                "max": ["river_storage", "protected_storage"], "min": ["flood_outflow"],
                "last": ["river_depth", "river_storage", "protected_storage"]}


def _value(model, name):
    b = model.base
    if name == "total_outflow":
        return b.river_outflow.double() + b.flood_outflow.double()
    return getattr(b, name).double()


def test_graph_statistics_equal_per_phase_replay(device):
    net = P.make_network("full", n=6000)
    kw = dict(variables_to_save=FLUX_DEPTH)
    g = P.model_for(net, **kw)
    h = P.model_for(net, **kw)
    spec = [(n, o) for o, names in FLUX_DEPTH.items() for n in names]
    acc = {}
    weight = 0.0
    for day in range(3):
        r = torch.as_tensor(syn.daily_runoff(net, day)[g.order]).to(device)
        g.set_inputs(r)
        g.step_advance()
        h.set_inputs(r)
        h.compute_adaptive_time_step()
        n = int(h.sub_step_counts()[0].item())
        dt = float(h.base.time_step[0].item())
        for k in range(n):
            for part in (_lib.PART_MOMENTUM, _lib.PART_LIMIT, _lib.PART_STAGE, _lib.PART_LEVEE):
                h.launch_substep_kernel(k, part)
            weight = weight + dt
            for name, op in spec:
                x = _value(h, name)
                key = f"{name}_{op}"
                if op == "mean":
                    acc[key] = acc.get(key, torch.zeros_like(x)) + x * dt
                elif op == "max":
                    a = acc.get(key, torch.full_like(x, -np.inf))
                    acc[key] = torch.where((x > a) | torch.isnan(x), x, a)
                elif op == "min":
                    a = acc.get(key, torch.full_like(x, np.inf))
                    acc[key] = torch.where((x < a) | torch.isnan(x), x, a)
        h.launch_substep_kernel(0, _lib.PART_END)
    got = g.collect_statistics()
    for name, op in spec:
        key = f"{name}_{op}"
        if op == "mean":
            # tensor / tensor: torch turns a division by a Python scalar into
            # a multiplication by its reciprocal
            ref = acc[key] / torch.full_like(acc[key], weight)
        else:
            ref = _value(h, name) if op == "last" else acc[key]
        assert torch.equal(got[key], ref), key
    # the state itself is unaffected by the statistics
    for k, v in g.state_tensors().items():
        assert torch.equal(v, h.state_tensors()[k]), k
    g.check_status()


@pytest.mark.parametrize("case", ["plain", "full"])
def test_statistics_match_oracle_fp64(case, device):
    net = P.make_network(case, n=5000)
    orc = P.oracle_for(net, "float64")
    P.spin_up(net, orc)
    spec_map = WITH_STORAGE if case == "full" else FLUX_DEPTH
    model = P.model_for(net, "float64", variables_to_save=spec_map)
    P.load_oracle_state(model, orc)
    spec = [(n, o) for o, names in spec_map.items() for n in names]
    replay = OF.StatsReplay(spec)

    def snap():
        s = orc.a
        out = {k: s[k] for k in P.CELL_REAL + P.CELL_STO}
        out["total_outflow"] = s["river_outflow"].astype(np.float64) + s["flood_outflow"]
        return out

    for day in range(2, 4):
        r = syn.daily_runoff(net, day)
        P.set_runoff_both(model, orc, r)
        model.step_advance()
        n = orc.adaptive_sub_steps(86400.0)
        orc.set_time_step(86400.0 / n)
        for _ in range(n):
            orc.substep()
            replay.add(snap(), orc.time_step)
    want = replay.result(snap())
    got = model.collect_statistics()
    order = model.order
    for key, ref in want.items():
        err = P.rel_err(got[key].cpu().numpy(), ref[order])
        assert err <= 1e-10, (key, err)


def test_ensemble_statistics_equal_single_member_runs(device):
    members = 4
    net = syn.generate_basins(40, 30_000, seed=9)
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=9)
    manning = (net.fields["river_manning"][:, None] * mfac).astype(np.float32)
    spec = {"mean": ["total_outflow", "river_storage"], "max": ["river_depth"], "last": ["flood_depth"]}
    mods = ["base", "adaptive_time"]
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods, num_members=members,
                    batched_fields={"river_manning": manning}, variables_to_save=spec)
    plains = []
    for m in range(members):
        f = dict(net.fields)
        f["river_manning"] = np.ascontiguousarray(manning[:, m])
        plains.append(CaMaFlood(device=device, input_proxy=f, opened_modules=mods, variables_to_save=spec))
    order = ens.order
    counts = []
    for day in range(2):
        r = syn.daily_runoff(net, day)
        rm = (r[:, None] * rfac).astype(np.float32)
        ens.set_inputs(torch.as_tensor(rm[order]).to(device))
        ens.step_advance()
        counts.append(ens.sub_step_counts().cpu().numpy().copy())
        for m, p in enumerate(plains):
            p.set_inputs(torch.as_tensor(np.ascontiguousarray(rm[:, m])[order]).to(device))
            p.step_advance()
    assert any(len(set(c.tolist())) > 1 for c in counts), counts   # members differ in dt
    a = ens.collect_statistics()
    for m, p in enumerate(plains):
        b = p.collect_statistics()
        for k in b:
            assert torch.equal(a[k][..., m], b[k]), (m, k)


def test_reset_and_periods(device):
    net = P.make_network("plain", n=3000)
    model = P.model_for(net, variables_to_save={"mean": ["total_outflow"], "last": ["river_depth"]})
    assert model.variables_to_save == {"mean": ["total_outflow"], "last": ["river_depth"]}
    r = torch.as_tensor(syn.daily_runoff(net, 0)[model.order]).to(device)
    model.set_inputs(r)
    model.step_advance()
    p1 = model.collect_statistics()          # resets
    model.step_advance()
    p2 = model.collect_statistics()
    assert not torch.equal(p1["total_outflow_mean"], p2["total_outflow_mean"])
    assert torch.equal(p2["river_depth_last"], model.base.river_depth.double())
    # a CTA-size change rebuilds the plan and keeps the statistics attached
    model._rebuild_plan(128)
    model.step_advance()
    p3 = model.collect_statistics()
    assert torch.isfinite(p3["total_outflow_mean"]).all()


def test_bad_specs_are_rejected(device):
    net = P.make_network("plain", n=500)
    with pytest.raises(ValueError):
        P.model_for(net, variables_to_save={"median": ["total_outflow"]})
    with pytest.raises(ValueError):
        P.model_for(net, variables_to_save={"mean": ["discharge"]})
    with pytest.raises(ValueError):
        P.model_for(net, variables_to_save={"mean": ["protected_depth"]})     # no levee module
