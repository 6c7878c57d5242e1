"""The PyTorch transcription of the reference step (oracle/step_torch.py),
the autograd oracle of the hand-written adjoint, pinned on the CPU:

* its forward equals the C oracle (oracle/cmf_oracle_impl.c, itself checked
  against outputs of the reference's CUDA kernels) in fp64 over a day of
  adaptive sub-steps;
* its autograd gradients equal central finite differences of its own
  forward for every differentiated input (h = 1e-4 relative, agreement
  within 1e-3 relative; central differences converge to the autograd value
  as h shrinks)."""
import numpy as np
import torch

from cmfb200 import synthetic as syn
from oracle import oracle as O, step_torch as ST

MODS = ["base", "adaptive_time"]


def _spun_up(n, seed, days=2):
    net = syn.generate(syn.NetworkSpec(n, seed=seed, levee_fraction=0.0))
    f = O.reference_fields(net.fields, MODS, "float64")
    orc = O.Oracle(f, MODS, "float64")
    for d in range(days):
        orc.set_runoff(syn.daily_runoff(net, d))
        orc.step_advance(86400.0, adaptive=True)
    return net, f, orc


def test_transcription_matches_c_oracle_fp64():
    net, f, orc = _spun_up(2000, seed=5)
    tr = ST.TorchRouting(f)
    st = orc.state()
    s = {k: torch.tensor(st[k], dtype=torch.float64) for k in ST.STATE}
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
    for k in ST.STATE:
        a, b = s[k].numpy(), o[k]
        err = np.max(np.abs(a - b) / (np.abs(b) + 1e-3 * np.mean(np.abs(b)) + 1e-300))
        assert err < 1e-9, (k, err)
    assert np.max(np.abs(ffr.numpy() - o["flood_fraction"])) < 1e-9


def test_transcription_autograd_matches_finite_differences():
    net, f, orc = _spun_up(300, seed=7)
    tr = ST.TorchRouting(f)
    st = orc.state()
    s0 = {k: torch.tensor(st[k], dtype=torch.float64) for k in ST.STATE}
    p0 = {k: torch.tensor(f[k], dtype=torch.float64) for k in ST.PARAMS}
    forcing = torch.tensor(np.stack([syn.daily_runoff(net, 2 + t) for t in range(2)]),
                           dtype=torch.float64)
    gauges = torch.arange(0, 300, 15)
    with torch.no_grad():
        truth = dict(p0, river_manning=p0["river_manning"] * 1.15)
        q_obs, _, _ = tr.window(s0, truth, forcing, 86400.0, gauges)

    def loss(p, forc):
        q, _, counts = tr.window(s0, p, forc, 86400.0, gauges)
        return ST.relative_misfit_loss(q, q_obs), counts

    p = {k: v.clone().requires_grad_(True) for k, v in p0.items()}
    fr = forcing.clone().requires_grad_(True)
    L, counts = loss(p, fr)
    grads = torch.autograd.grad(L, [p[k] for k in ST.PARAMS] + [fr])
    for name, g in zip(list(ST.PARAMS) + ["runoff"], grads):
        flat = g[0] if name == "runoff" else g
        for c in torch.argsort(flat.abs(), descending=True)[:3].tolist():
            vals = []
            for sign in (1, -1):
                pp = {k: v.clone() for k, v in p0.items()}
                ff = forcing.clone()
                tgt = ff[0] if name == "runoff" else pp[name]
                h = 1e-4 * abs(tgt[c].item())
                tgt[c] += sign * h
                with torch.no_grad():
                    l, cc = loss(pp, ff)
                assert cc == counts
                vals.append(l.item())
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(flat[c].item() - fd) <= 1e-3 * abs(fd), (name, c, flat[c].item(), fd)
