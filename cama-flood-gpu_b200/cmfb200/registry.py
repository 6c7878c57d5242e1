"""Reference-facing backend: the per-interval step of a reference model run
by this library.

The reference dispatches its physics through registries
(`BackendRegistry({"metal", "cuda", "triton"}, name, spec).selected`,
cmfgpu/phys/outflow.py:51-60) and advances an interval with the sub-step
loop of `CaMaFlood.step_advance` (cmfgpu/models/cama_flood_model.py:104-173).
`B200Backend` is the object a "b200" registry entry would return: built once
from the reference model's tensors, then `set_inputs` / `step_advance` per
interval, with every array in the REFERENCE model's catchment order.

This library routes in its own catchment order (breadth-first from the
mouths, so that each catchment's upstream cells are contiguous).  The
adapter owns that permutation: runoff handed in reference order is permuted
on the device before each interval, and `state()` / `write_back()` hand the
state back in reference order.  A caller therefore never sees the internal
order, and forcing mapped with the reference's own catchment ids lands on the
right cells.
"""
from __future__ import annotations

from typing import Iterable, Mapping, Optional

import numpy as np
import torch

from .model import CaMaFlood


class B200Backend:
    """Interval step of a reference model on libcmfb200.

    `fields` maps the reference's field names to arrays or tensors in the
    reference model's catchment order (what its modules hold: catchment_id,
    downstream_id, river_width, ..., the state tensors); `opened_modules` is
    the reference model's list.  Keyword arguments go to `CaMaFlood`
    (step_duration, precision, BLOCK_SIZE, ...)."""

    def __init__(self, fields: Mapping[str, object], opened_modules: Iterable[str],
                 device: str | torch.device = "cuda", **model_kw):
        host = {k: (v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v))
                for k, v in fields.items()}
        self.model = CaMaFlood(device=device, input_proxy=host, opened_modules=opened_modules,
                               **model_kw)

    @property
    def catchment_id(self) -> np.ndarray:
        """Catchment ids in the reference order (the order of every array the
        adapter takes or returns)."""
        return self.model.base.catchment_id.cpu().numpy()[self.model.inverse_order]

    @property
    def state_names(self) -> list[str]:
        """Names of the state tensors the interval step updates."""
        return list(self.model.state_tensors())

    def set_inputs(self, runoff, inflow=None, sea_surface_elevation=None) -> None:
        """Runoff [N] (or [N, M]) in m^3/s, reference catchment order."""
        self.model.set_inputs(runoff, inflow, sea_surface_elevation, order="input")

    def step_advance(self, num_sub_steps: Optional[int] = None) -> None:
        self.model.step_advance(num_sub_steps)

    def state(self, names: Optional[Iterable[str]] = None) -> dict[str, torch.Tensor]:
        """State tensors in reference catchment order (copies)."""
        return self.model.read_state(names, order="input")

    def write_back(self, targets: Mapping[str, torch.Tensor]) -> None:
        """Copy the state into the reference model's own tensors (reference
        order), e.g. before its output writers read them."""
        for k, v in self.state(list(targets)).items():
            targets[k].copy_(v.to(targets[k].dtype))

    def close(self) -> None:
        self.model.close()
