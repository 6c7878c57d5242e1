"""The CPU oracle against golden fixtures made by the reference's own CUDA
kernels on a B200 (tests/golden/make_ref_golden.py): the CFL sub-step count
and dt exactly, one sub-step within 1e-4 relative (max over cells; the oracle
rounds every float operation once while nvcc contracts to FMA) with >= 95 % of
values bit-identical or within 1e-5.  This pins the oracle to the reference."""
from pathlib import Path

import numpy as np
import pytest

from cmfb200 import synthetic as syn
from oracle import oracle as O

import golden_cases as G

GOLD = Path(__file__).parent / "golden"


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    floor = max(1e-3 * float(np.mean(np.abs(b))), 1e-30)
    return np.abs(a - b) / (np.abs(b) + floor)


@pytest.mark.parametrize("case", list(G.CASES))
def test_oracle_matches_reference_golden(case):
    path = GOLD / f"ref_{case}.npz"
    if not path.exists():
        pytest.skip("fixture not generated")
    g = np.load(path)
    net = syn.generate(G.CASES[case])
    f = O.reference_fields(net.fields, net.opened_modules)
    for k in G.state_fields(net.opened_modules):
        f[k] = g["in_" + k]
    orc = O.Oracle(f, net.opened_modules)
    O.set_threads(1)
    orc.set_runoff(syn.daily_runoff(net, 1))
    n = orc.adaptive_sub_steps(86400.0)
    assert n == int(g["n"])
    orc.set_time_step(86400.0 / n)
    assert np.float32(orc.time_step) == g["dt"]
    orc.substep()
    for k in G.state_fields(net.opened_modules) + ["river_inflow", "flood_inflow"]:
        r = _rel(orc.a[k], g["out_" + k])
        assert r.max() <= 1e-4, (k, float(r.max()))
        assert np.mean(r <= 1e-5) >= 0.95, (k, float(np.mean(r <= 1e-5)))
