"""Hand-written CUDA adjoint of the sub-step (cmfb200.adjoint) against
autograd through the PyTorch transcription of the reference step
(oracle/step_torch.py) and against central finite differences, for the base
physics and for full physics (bifurcation paths, levees, reservoirs).

Setting: an fp64 network, a window of daily intervals with adaptive
sub-steps, discharge observed at gauges, loss = sum of squared relative
misfit against a run with perturbed river Manning n.  Checkpoint segments
are made short so that segments cross interval boundaries."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn, topology
from cmfb200.adjoint import AdjointRouting, PARAMS
from oracle import step_torch as ST

pytestmark = pytest.mark.gpu

DAYS = 2
CASES = {"plain": dict(levee_fraction=0.0),
         "full": dict(bifurcation_paths=40, levee_fraction=0.25, reservoirs=10)}
STATIC = ("downstream_idx", "river_length", "catchment_elevation", "catchment_area",
          "downstream_distance", "flood_depth_table", "levee_catchment_idx",
          "levee_crown_height", "levee_fraction", "levee_base_height",
          "reservoir_catchment_idx", "conservation_volume", "emergency_volume",
          "adjustment_volume", "effective_normal_outflow", "adjustment_outflow",
          "flood_control_outflow", "is_reservoir", "is_dam_upstream", "is_dam_related",
          "bifurcation_catchment_idx", "bifurcation_downstream_idx", "bifurcation_manning",
          "bifurcation_width", "bifurcation_length", "bifurcation_elevation")


def _setup(device, case="plain", n=1500, seed=13, checkpoint_every=50):
    net = syn.generate(syn.NetworkSpec(n, seed=seed, **CASES[case]))
    model = CaMaFlood(device=device, input_proxy=net.fields,
                      opened_modules=net.opened_modules, precision="float64")
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


@pytest.mark.parametrize("case", ["plain", "full"])
def test_primal_matches_product_forward(case, device):
    net, model, eng, forcing = _setup(device, case)
    params = eng.parameters()
    state0 = eng.initial_state()
    _, final = eng.forward_only(params, forcing, state0)
    for d in range(DAYS):
        model.set_inputs(forcing[d])
        model.step_advance()
    ref = eng.unpack(eng.initial_state())
    got = eng.unpack(final)
    for name in ref:
        a, b = got[name].cpu().numpy(), ref[name].cpu().numpy()
        if name == "protected_depth":            # only levee cells carry it
            mask = np.zeros(eng.N, dtype=bool)
            if model.levee is not None:
                mask[model.levee.levee_catchment_idx.cpu().numpy()] = True
            a, b = a[mask], b[mask]
        if b.size == 0:
            continue
        scale = np.abs(b).mean() + 1e-300
        err = np.max(np.abs(a - b)) / scale
        assert err < 1e-12, (name, err)


@pytest.mark.parametrize("case", ["plain", "full"])
def test_gradients_match_transcription_autograd(case, device):
    net, model, eng, forcing = _setup(device, case)
    params = eng.parameters()
    state0 = eng.initial_state()
    q_obs = _observed(eng, params, forcing, state0)

    # CUDA adjoint
    p = {k: v.clone().requires_grad_(True) for k, v in params.items()}
    forc = forcing.clone().requires_grad_(True)
    s0 = state0.clone().requires_grad_(True)
    q, _ = eng.window(p, forc, s0)
    g_cuda = torch.autograd.grad(_loss(q, q_obs), [p[k] for k in PARAMS] + [forc, s0])

    # autograd through the transcription (CPU, fp64, same model order)
    fx = model.export_fields()
    tr = ST.TorchRouting({k: fx[k] for k in STATIC if k in fx}, net.opened_modules)
    pt = {k: v.detach().cpu().clone().requires_grad_(True) for k, v in params.items()}
    ft = forcing.detach().cpu().clone().requires_grad_(True)
    sv = {k: v.detach().cpu() for k, v in eng.unpack(state0).items()}
    st0 = {k: sv[k].clone().requires_grad_(True) for k in tr.names}
    qt, _, counts = tr.window(st0, pt, ft, eng.outer, eng.gauges.cpu())
    assert torch.allclose(qt, q.detach().cpu(), rtol=1e-10, atol=0)
    inputs = [pt[k] for k in PARAMS] + [ft] + [st0[k] for k in tr.names]
    g_ref = torch.autograd.grad(_loss(qt, q_obs.cpu()), inputs, allow_unused=True)
    g_ref = [torch.zeros_like(x) if g is None else g for x, g in zip(inputs, g_ref)]

    s_cuda = {k: v.cpu().numpy() for k, v in eng.unpack(g_cuda[5]).items()}
    pairs = list(zip(list(PARAMS) + ["runoff"], g_cuda[:5], g_ref[:5]))
    pairs += [("state0:" + k, s_cuda[k], g) for k, g in zip(tr.names, g_ref[5:])]
    pairs = [(name, np.asarray(a.detach().cpu() if torch.is_tensor(a) else a).ravel(),
              b.detach().cpu().numpy().ravel()) for name, a, b in pairs]
    overall = max(np.abs(b).max() for _, _, b in pairs)
    for name, a, b in pairs:
        # a field whose gradient is zero in the transcription is held to the
        # scale of the largest gradient (rounding-level residue allowed)
        scale = max(np.abs(b).max(), 1e-12 * overall)
        err = np.max(np.abs(a - b)) / scale
        assert err < 1e-8, (name, err)


@pytest.mark.parametrize("case", ["plain", "full"])
def test_gradients_match_finite_differences(case, device):
    net, model, eng, forcing = _setup(device, case, n=2000, seed=17)
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

    def fd(name, c, h_rel):
        h = h_rel * abs(forcing[0, c].item() if name == "runoff" else params[name][c].item())
        vals = []
        for sign in (1, -1):
            pp = {k: v.clone() for k, v in params.items()}
            ff = forcing.clone()
            if name == "runoff":
                ff[0, c] += sign * h
            else:
                pp[name][c] += sign * h
            vals.append(loss_at(pp, ff))
        return (vals[0] - vals[1]) / (2 * h)

    # h = 1e-4 relative; where that step crosses a branch of the piecewise
    # physics (levee cases, flood levels) the difference is retaken at 1e-6
    for name, g in zip(list(PARAMS) + ["runoff"], grads):
        flat = (g[0] if name == "runoff" else g).detach()
        for c in torch.argsort(flat.abs(), descending=True)[:5].tolist():
            ad = flat[c].item()
            ok = any(abs(ad - fd(name, c, h)) <= 1e-3 * abs(ad) for h in (1e-4, 1e-6))
            assert ok, (name, c, ad, fd(name, c, 1e-4), fd(name, c, 1e-6))


def test_gradients_match_finite_differences_random_cells(device):
    """The benchmark definition's check at reduced size: central differences
    at 50 random cells per parameter (river and floodplain Manning, river
    height, river width, runoff of the first day), full physics, fp64.  A cell
    matches when |ad - fd| <= 1e-3 * max(|ad|, 1e-3 * max|grad of that field|)
    at h = 1e-4 relative, or at h = 1e-6 where the larger step crosses a branch
    of the piecewise physics."""
    net, model, eng, forcing = _setup(device, "full", n=4000, seed=29)
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

    def fd(name, c, h_rel):
        base = forcing[0, c].item() if name == "runoff" else params[name][c].item()
        h = h_rel * abs(base)
        if h == 0.0:
            return 0.0
        vals = []
        for sign in (1, -1):
            pp = {k: v.clone() for k, v in params.items()}
            ff = forcing.clone()
            if name == "runoff":
                ff[0, c] += sign * h
            else:
                pp[name][c] += sign * h
            vals.append(loss_at(pp, ff))
        return (vals[0] - vals[1]) / (2 * h)

    rng = np.random.default_rng(29)
    failures = []
    for name, g in zip(list(PARAMS) + ["runoff"], grads):
        flat = (g[0] if name == "runoff" else g).detach()
        gmax = float(flat.abs().max())
        for c in rng.choice(eng.N, size=50, replace=False).tolist():
            ad = flat[c].item()
            tol = 1e-3 * max(abs(ad), 1e-3 * gmax)
            if not any(abs(ad - fd(name, c, h)) <= tol for h in (1e-4, 1e-6)):
                failures.append((name, c, ad, fd(name, c, 1e-4), fd(name, c, 1e-6)))
    assert not failures, failures[:5]
