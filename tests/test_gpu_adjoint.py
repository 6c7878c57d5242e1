"""Hand-written CUDA adjoint of the sub-step (cmfb200.adjoint) against
autograd through the PyTorch transcription of the reference step
(oracle/step_torch.py) and against central finite differences.

Setting: a base-physics network in fp64, a window of daily intervals with
adaptive sub-steps, discharge observed at gauges, loss = sum of squared
relative misfit against a run with perturbed river Manning n.  Checkpoint
segments are made short so that segments cross interval boundaries."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn, topology
from cmfb200.adjoint import AdjointRouting, PARAMS, STATE
from oracle import step_torch as ST

pytestmark = pytest.mark.gpu

DAYS = 2


def _setup(device, n=1500, seed=13, checkpoint_every=50):
    net = syn.generate(syn.NetworkSpec(n, seed=seed, levee_fraction=0.0))
    model = CaMaFlood(device=device, input_proxy=net.fields,
                      opened_modules=["base", "adaptive_time"], precision="float64")
    for d in range(2):                                   # spin up
        model.set_inputs(torch.as_tensor(syn.daily_runoff(net, d)[model.order]).to(device))
        model.step_advance()
    fx = model.export_fields()
    area = topology.accumulate_upstream(fx["downstream_idx"], fx["catchment_area"].astype(np.float64))
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(area > np.quantile(area, 0.8))
    gauges = np.sort(rng.choice(cand, size=min(40, cand.size), replace=False))
    eng = AdjointRouting(model, gauges, checkpoint_every=checkpoint_every)
    forcing = torch.as_tensor(np.stack([syn.daily_runoff(net, 2 + d)[model.order]
                                        for d in range(DAYS)]), dtype=torch.float64, device=device)
    return net, model, eng, forcing


def _observed(eng, params, forcing, state0, seed=5):
    rng = np.random.default_rng(seed)
    truth = dict(params)
    fac = torch.as_tensor(np.exp(0.2 * rng.standard_normal(eng.N)), device=eng.device)
    truth["river_manning"] = params["river_manning"] * fac
    q_obs, _ = eng.forward_only(truth, forcing, state0)
    return q_obs


def _loss(q, q_obs):
    return (((q - q_obs) / q_obs) ** 2).sum()


def test_primal_matches_product_forward(device):
    net, model, eng, forcing = _setup(device)
    params = eng.parameters()
    state0 = eng.initial_state()
    _, final = eng.forward_only(params, forcing, state0)
    for d in range(DAYS):
        model.set_inputs(forcing[d])
        model.step_advance()
    ref = eng.initial_state()
    for k, name in enumerate(STATE):
        a, b = final[k].cpu().numpy(), ref[k].cpu().numpy()
        scale = np.abs(b).mean() + 1e-300
        err = np.max(np.abs(a - b)) / scale
        assert err < 1e-12, (name, err)


def test_gradients_match_transcription_autograd(device):
    net, model, eng, forcing = _setup(device)
    params = eng.parameters()
    state0 = eng.initial_state()
    q_obs = _observed(eng, params, forcing, state0)

    # CUDA adjoint
    p = {k: v.clone().requires_grad_(True) for k, v in params.items()}
    forc = forcing.clone().requires_grad_(True)
    s0 = state0.clone().requires_grad_(True)
    q, _ = eng.window(p, forc, s0)
    loss = _loss(q, q_obs)
    g_cuda = torch.autograd.grad(loss, [p[k] for k in PARAMS] + [forc, s0])

    # autograd through the transcription (CPU, fp64, same model order)
    fx = model.export_fields()
    tr = ST.TorchRouting({k: fx[k] for k in ("downstream_idx", "river_length",
                                            "catchment_elevation", "catchment_area",
                                            "downstream_distance", "flood_depth_table")})
    pt = {k: v.detach().cpu().clone().requires_grad_(True) for k, v in params.items()}
    ft = forcing.detach().cpu().clone().requires_grad_(True)
    st0 = state0.detach().cpu().clone().requires_grad_(True)
    s_dict = {k: st0[i] for i, k in enumerate(STATE)}
    qt, _, counts = tr.window(s_dict, pt, ft, eng.outer, eng.gauges.cpu())
    assert torch.allclose(qt, q.detach().cpu(), rtol=1e-10, atol=0)
    lt = _loss(qt, q_obs.cpu())
    g_ref = torch.autograd.grad(lt, [pt[k] for k in PARAMS] + [ft, st0])

    names = list(PARAMS) + ["runoff", "state0"]
    for name, a, b in zip(names, g_cuda, g_ref):
        a = a.detach().cpu().numpy().ravel()
        b = b.detach().cpu().numpy().ravel()
        scale = np.abs(b).max()
        assert scale > 0, name
        err = np.max(np.abs(a - b)) / scale
        assert err < 1e-8, (name, err)


def test_gradients_match_finite_differences(device):
    net, model, eng, forcing = _setup(device, n=2000, seed=17)
    params = eng.parameters()
    state0 = eng.initial_state()
    q_obs = _observed(eng, params, forcing, state0)
    p = {k: v.clone().requires_grad_(True) for k, v in params.items()}
    forc = forcing.clone().requires_grad_(True)
    q, _ = eng.window(p, forc, state0)
    grads = torch.autograd.grad(_loss(q, q_obs), [p[k] for k in PARAMS] + [forc])

    def loss_at(pp, ff):
        qq, _ = eng.forward_only(pp, ff, state0)
        return float(_loss(qq, q_obs))

    h_rel = 1e-4
    for name, g in zip(list(PARAMS) + ["runoff"], grads):
        g = g.detach()
        flat = g[0] if name == "runoff" else g
        cells = torch.argsort(flat.abs(), descending=True)[:6].tolist()
        for c in cells:
            if name == "runoff":
                base = forcing[0, c].item()
            else:
                base = params[name][c].item()
            h = h_rel * abs(base)

            def perturbed(sign):
                pp = {k: v.clone() for k, v in params.items()}
                ff = forcing.clone()
                if name == "runoff":
                    ff[0, c] += sign * h
                else:
                    pp[name][c] += sign * h
                return loss_at(pp, ff)

            fd = (perturbed(1) - perturbed(-1)) / (2 * h)
            ad = flat[c].item()
            assert abs(ad - fd) <= 1e-3 * abs(fd) + 1e-12, (name, c, ad, fd)
