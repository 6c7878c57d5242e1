"""Error of every output of the mixed-precision path (fp32 fluxes, fp64
storage -- the reference's default) against an fp64 oracle run of the same
inputs and sub-step counts, one simulated day.

The product is bit-identical to the reference's own CUDA kernels
(test_gpu_parity.py), so these figures are also the reference's error.  The
test prints the per-field table (pytest -s) and holds it under stated bounds:
max relative error (floor 1e-3 of the field's mean magnitude) and the 99th
percentile of the per-cell relative error."""
import numpy as np
import pytest
import torch

from cmfb200 import synthetic as syn
import parity as P

pytestmark = pytest.mark.gpu

# bounds on (max, p99) relative error after one day
BOUNDS = {"storage": (2e-3, 1e-4), "other": (3e-2, 1e-3)}


def _p99(a, b, floor_frac=1e-3):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    floor = max(float(np.mean(np.abs(b))) * floor_frac, 1e-30)
    return float(np.quantile(np.abs(a - b) / (np.abs(b) + floor), 0.99))


@pytest.mark.parametrize("case", ["plain", "full"])
def test_mixed_precision_error_vs_fp64_oracle(case, device):
    net = P.make_network(case, n=6000, seed=23)
    model = P.model_for(net, "float32")
    orc = P.oracle_for(net, "float64")
    for d in range(2):
        r = syn.daily_runoff(net, d)
        model.set_inputs(torch.as_tensor(r[model.order]).to(device))
        model.step_advance()
        n = int(model.sub_step_counts()[0].item())
        orc.set_runoff(r)
        orc.step_advance(86400.0, adaptive=False, fixed_n=n)
    torch.cuda.synchronize()
    order = model.order
    rows = []
    for k in P.CELL_REAL + P.CELL_STO:
        a = getattr(model.base, k).cpu().numpy()
        b = orc.a[k][order]
        rows.append((k, P.rel_err(a, b), _p99(a, b)))
    if model.bifurcation is not None:
        for k in P.PATH_FIELDS:
            a = getattr(model.bifurcation, k).cpu().numpy()
            rows.append((k, P.rel_err(a, orc.a[k]), _p99(a, orc.a[k])))
    print(f"\n{case}: mixed precision vs fp64 oracle after 2 days (max rel, p99 rel)")
    for k, mx, p in rows:
        print(f"  {k:36s} {mx:9.2e} {p:9.2e}")
    for k, mx, p in rows:
        bmax, bp99 = BOUNDS["storage" if k.endswith("storage") else "other"]
        assert mx < bmax and p < bp99, (k, mx, p)
