"""Helpers shared by the GPU parity tests (test infrastructure).

A case is a seeded synthetic network.  The product model runs it in its own
breadth-first catchment order; the oracle runs the same inputs in the
generator's original order.  Fields are compared after mapping through
`model.order` (model index -> input index); bifurcation paths keep their order.
"""
from __future__ import annotations

import numpy as np
import torch

from cmfb200 import CaMaFlood, synthetic as syn
from oracle import oracle as O

CELL_REAL = ("river_outflow", "flood_outflow", "river_depth", "flood_depth", "protected_depth",
             "river_cross_section_depth", "flood_cross_section_depth", "flood_cross_section_area",
             "flood_fraction")
CELL_STO = ("river_storage", "flood_storage", "protected_storage")
PATH_FIELDS = ("bifurcation_outflow", "bifurcation_cross_section_depth")

CASES = {
    "plain": dict(levee_fraction=0.0),
    "bif": dict(bifurcation_paths=300),
    "levee": dict(levee_fraction=0.25),
    "res": dict(reservoirs=30),
    "full": dict(bifurcation_paths=300, levee_fraction=0.25, reservoirs=30),
}


def make_network(case: str, n: int = 6000, seed: int = 21) -> syn.Network:
    return syn.generate(syn.NetworkSpec(n, seed=seed, **CASES[case]))


def oracle_for(net: syn.Network, precision="float32") -> O.Oracle:
    f = O.reference_fields(net.fields, net.opened_modules, precision)
    return O.Oracle(f, net.opened_modules, precision)


def model_for(net: syn.Network, precision="float32", **kw) -> CaMaFlood:
    return CaMaFlood(device="cuda:0", input_proxy=net.fields, opened_modules=net.opened_modules,
                     precision=precision, **kw)


def spin_up(net: syn.Network, orc: O.Oracle, days: int = 2, outer=86400.0) -> None:
    for d in range(days):
        orc.set_runoff(syn.daily_runoff(net, d))
        orc.step_advance(outer, adaptive=True)


def load_oracle_state(model: CaMaFlood, orc: O.Oracle) -> None:
    """Copy the oracle state (input order) into the model tensors (model order)."""
    order = model.order
    s = orc.a
    b = model.base
    for k in CELL_REAL + CELL_STO:
        getattr(b, k).copy_(torch.as_tensor(s[k][order]))
    if model.bifurcation is not None:
        for k in PATH_FIELDS:
            getattr(model.bifurcation, k).copy_(torch.as_tensor(s[k]))
    if model.reservoir is not None:
        model.reservoir.reservoir_total_inflow.copy_(torch.as_tensor(s["reservoir_total_inflow"][order]))


def set_runoff_both(model: CaMaFlood, orc: O.Oracle, runoff: np.ndarray) -> None:
    orc.set_runoff(runoff)
    model.set_inputs(torch.as_tensor(runoff[model.order]).to(model.device))


def rel_err(a: np.ndarray, b: np.ndarray, floor_frac: float = 1e-3) -> float:
    """max |a-b| / (|b| + floor), floor = floor_frac * mean|b| (scale of the field)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    scale = float(np.mean(np.abs(b))) if b.size else 0.0
    floor = max(scale * floor_frac, 1e-30)
    return float(np.max(np.abs(a - b) / (np.abs(b) + floor)))


def compare(model: CaMaFlood, orc: O.Oracle, diag: bool = True) -> dict[str, float]:
    """Per-field max relative error of the model against the oracle."""
    order = model.order
    out = {}
    s = orc.a
    b = model.base
    for k in CELL_REAL + CELL_STO:
        out[k] = rel_err(getattr(b, k).cpu().numpy(), s[k][order])
    if model.bifurcation is not None:
        for k in PATH_FIELDS:
            out[k] = rel_err(getattr(model.bifurcation, k).cpu().numpy(), s[k])
    if model.reservoir is not None:
        out["reservoir_total_inflow"] = rel_err(model.reservoir.reservoir_total_inflow.cpu().numpy(),
                                                s["reservoir_total_inflow"][order])
    if diag:
        out["river_inflow"] = rel_err(b.river_inflow.cpu().numpy(), s["river_inflow"][order])
        out["flood_inflow"] = rel_err(b.flood_inflow.cpu().numpy(), s["flood_inflow"][order])
        if model.bifurcation is not None:
            out["limit_rate"] = rel_err(model.bifurcation.limit_rate.cpu().numpy(), s["limit_rate"][order])
            out["global_bifurcation_outflow"] = rel_err(
                model.bifurcation.global_bifurcation_outflow.cpu().numpy(),
                s["global_bifurcation_outflow"][order])
            out["water_surface_elevation"] = rel_err(b.water_surface_elevation.cpu().numpy(),
                                                     s["water_surface_elevation"][order])
        if b.total_storage is not None:
            out["total_storage"] = rel_err(b.total_storage.cpu().numpy(), s["total_storage"][order])
        if b.protected_water_surface_elevation is not None:
            out["protected_water_surface_elevation"] = rel_err(
                b.protected_water_surface_elevation.cpu().numpy(),
                s["protected_water_surface_elevation"][order])
    return out


def mismatch_fraction(model: CaMaFlood, orc: O.Oracle, rtol: float = 1e-5) -> dict[str, float]:
    """Fraction of cells whose relative error exceeds rtol (per field)."""
    order = model.order
    s = orc.a
    out = {}
    for k in CELL_REAL + CELL_STO:
        a = getattr(model.base, k).cpu().numpy().astype(np.float64)
        r = s[k][order].astype(np.float64)
        floor = max(1e-3 * float(np.mean(np.abs(r))), 1e-30)
        out[k] = float(np.mean(np.abs(a - r) > rtol * (np.abs(r) + floor)))
    return out


def ref_cuda_from_oracle(net: syn.Network, orc: O.Oracle):
    """The reference's CUDA kernels (oracle/_ref) loaded with the oracle's
    current state."""
    from oracle import ref_cuda as RC
    f = O.reference_fields(net.fields, net.opened_modules)
    st = orc.state()
    f.update({k: st[k] for k in CELL_REAL + CELL_STO})
    if "bifurcation" in net.opened_modules:
        f.update({k: st[k] for k in PATH_FIELDS})
    if "reservoir" in net.opened_modules:
        f["reservoir_total_inflow"] = st["reservoir_total_inflow"]
    return RC.RefCuda(f, net.opened_modules)


def assert_bit_exact(model: CaMaFlood, ref_state: dict, diag: bool) -> None:
    """Every state field of the model equals the reference CUDA state."""
    order = model.order
    for k in CELL_REAL + CELL_STO:
        np.testing.assert_array_equal(getattr(model.base, k).cpu().numpy(), ref_state[k][order],
                                      err_msg=k)
    if model.bifurcation is not None:
        for k in PATH_FIELDS:
            np.testing.assert_array_equal(getattr(model.bifurcation, k).cpu().numpy(),
                                          ref_state[k], err_msg=k)
    if model.reservoir is not None:
        np.testing.assert_array_equal(model.reservoir.reservoir_total_inflow.cpu().numpy(),
                                      ref_state["reservoir_total_inflow"][order])
    if diag:
        for k in ("river_inflow", "flood_inflow"):
            np.testing.assert_array_equal(getattr(model.base, k).cpu().numpy(),
                                          ref_state[k][order], err_msg=k)
