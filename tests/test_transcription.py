"""The PyTorch transcription of the reference step (oracle/step_torch.py),
the autograd oracle of the hand-written adjoint, pinned on the CPU:

* its forward equals the C oracle (oracle/cmf_oracle_impl.h, itself checked
  against outputs of the reference's CUDA kernels) in fp64 over a day of
  adaptive sub-steps, for every physics combination;
* its autograd gradients equal central finite differences of its own
  forward for every differentiated input, base and full physics.  The step
  is h = 1e-4 relative as the calibration check prescribes; where that step
  crosses a branch of the piecewise physics (levee cases, flood levels) the
  difference is retaken at h = 1e-6, which converges to the autograd value.
"""
import numpy as np
import pytest
import torch

from cmfb200 import synthetic as syn
from oracle import oracle as O, step_torch as ST
import parity as P


def _spun_up(net, days=2):
    mods = net.opened_modules
    f = O.reference_fields(net.fields, mods, "float64")
    orc = O.Oracle(f, mods, "float64")
    for d in range(days):
        orc.set_runoff(syn.daily_runoff(net, d))
        orc.step_advance(86400.0, adaptive=True)
    return f, orc


@pytest.mark.parametrize("case", ["plain", "bif", "levee", "res", "full"])
def test_transcription_matches_c_oracle_fp64(case):
    net = P.make_network(case, n=2000, seed=5)
    f, orc = _spun_up(net)
    tr = ST.TorchRouting(f, net.opened_modules)
    st = orc.state()
    s = {k: torch.tensor(st[k], dtype=torch.float64) for k in tr.names}
    p = {k: torch.tensor(f[k], dtype=torch.float64) for k in ST.PARAMS}
    n = orc.adaptive_sub_steps(86400.0)
    assert tr.sub_steps(s, 86400.0) == n
    r = syn.daily_runoff(net, 2)
    orc.set_runoff(r)
    orc.set_time_step(86400.0 / n, 86400.0)
    rt = torch.tensor(r, dtype=torch.float64)
    for _ in range(n):
        orc.substep()
        s, ffr = tr.substep(s, p, rt, 86400.0 / n)
    o = orc.state()
    for k in tr.names:
        a, b = s[k].numpy(), o[k]
        err = np.max(np.abs(a - b) / (np.abs(b) + 1e-3 * np.mean(np.abs(b)) + 1e-300))
        assert err < 1e-9, (k, err)
    assert np.max(np.abs(ffr.numpy() - o["flood_fraction"])) < 1e-9


@pytest.mark.parametrize("case", ["plain", "full"])
def test_transcription_autograd_matches_finite_differences(case):
    extra = dict(levee_fraction=0.0) if case == "plain" else dict(
        bifurcation_paths=40, levee_fraction=0.3, reservoirs=8)
    net = syn.generate(syn.NetworkSpec(400, seed=9, **extra))
    f, orc = _spun_up(net)
    tr = ST.TorchRouting(f, net.opened_modules)
    st = orc.state()
    s0 = {k: torch.tensor(st[k], dtype=torch.float64) for k in tr.names}
    p0 = {k: torch.tensor(f[k], dtype=torch.float64) for k in ST.PARAMS}
    forcing = torch.tensor(np.stack([syn.daily_runoff(net, 2 + t) for t in range(1)]),
                           dtype=torch.float64)
    gauges = torch.arange(0, 400, 10)
    with torch.no_grad():
        truth = dict(p0, river_manning=p0["river_manning"] * 1.15)
        q_obs, _, _ = tr.window(s0, truth, forcing, 86400.0, gauges)

    def loss(p, forc, s):
        q, _, counts = tr.window(s, p, forc, 86400.0, gauges)
        return ST.relative_misfit_loss(q, q_obs), counts

    p = {k: v.clone().requires_grad_(True) for k, v in p0.items()}
    fr = forcing.clone().requires_grad_(True)
    sd = {k: v.clone().requires_grad_(True) for k, v in s0.items()}
    L, counts = loss(p, fr, sd)
    checked = list(ST.PARAMS) + ["runoff", "river_storage", "river_depth", "river_outflow"]
    if case == "full":
        checked += ["bifurcation_outflow", "bifurcation_cross_section_depth"]
    inputs = [p[k] for k in ST.PARAMS] + [fr] + [sd[k] for k in checked[5:]]
    grads = torch.autograd.grad(L, inputs)

    def fd(name, c, h_rel):
        vals = []
        for sign in (1, -1):
            pp = {k: v.clone() for k, v in p0.items()}
            ff = forcing.clone()
            ss = {k: v.clone() for k, v in s0.items()}
            tgt = ff[0] if name == "runoff" else (pp[name] if name in p0 else ss[name].reshape(-1))
            h = h_rel * abs(tgt[c].item())
            tgt[c] += sign * h
            with torch.no_grad():
                l, cc = loss(pp, ff, ss)
            assert cc == counts
            vals.append(l.item())
        return (vals[0] - vals[1]) / (2 * h)

    for name, g in zip(checked, grads):
        flat = g[0] if name == "runoff" else g.reshape(-1)
        for c in torch.argsort(flat.abs(), descending=True)[:2].tolist():
            ad = flat[c].item()
            ok = any(abs(ad - fd(name, c, h)) <= 1e-3 * abs(ad) for h in (1e-4, 1e-6))
            assert ok, (name, c, ad, fd(name, c, 1e-4), fd(name, c, 1e-6))
