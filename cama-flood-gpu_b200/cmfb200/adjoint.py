"""Differentiable routing windows over the hand-written CUDA adjoint.

`RoutingWindow` is a `torch.autograd.Function`: its forward runs a window of
forcing intervals through the fp64 primal kernels of libcmfb200
(`cmf_adj_forward`), storing the state every `checkpoint_every` sub-steps;
its backward recomputes each checkpoint segment with a tape and sweeps it in
reverse (`cmf_adj_reverse`).  The gradients reach the river and floodplain
Manning coefficients, river height, river width, the runoff of every interval
and the initial state.  Every physics module of the model is differentiated:
base, bifurcation, levee and reservoir.

The sub-step counts of the intervals come from the CFL rule on the state at
each interval start (cmfgpu/phys/cuda/adaptive_time.cu:19-48) and carry no
gradient, like `floor` and `.item()` in the reference's step
(cmfgpu/models/cama_flood_model.py:119-132).

State: one flat fp64 tensor, model (breadth-first) order: the cell fields
`CELL_STATE` as [12, N], then the path fields `PATH_STATE` as [2, P*L]
(`AdjointRouting.unpack` / `pack` convert).  Parameters and forcing are
model-ordered fp64 tensors.
"""
from __future__ import annotations

import bisect
import ctypes

import torch

from . import _lib

CELL_STATE = ("river_storage", "flood_storage", "river_outflow", "flood_outflow", "river_depth",
              "flood_depth", "river_cross_section_depth", "flood_cross_section_depth",
              "flood_cross_section_area", "protected_storage", "protected_depth",
              "reservoir_total_inflow")
PATH_STATE = ("bifurcation_outflow", "bifurcation_cross_section_depth")
STATE = CELL_STATE + PATH_STATE
PARAMS = ("river_manning", "flood_manning", "river_height", "river_width")
F_ROUT, F_FOUT = 2, 3
SLOT_CELL_FIELDS = 15        # the 12 cell state fields + flux, flux, limit rate


def _bind(h) -> None:
    if getattr(h, "_adj_bound", False):
        return
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    I64 = ctypes.c_int64
    h.cmf_adj_sizes.restype = I
    h.cmf_adj_sizes.argtypes = [P, ctypes.POINTER(I64), ctypes.POINTER(I64), ctypes.POINTER(I64),
                                ctypes.POINTER(I)]
    h.cmf_adj_plan_create.restype = I
    h.cmf_adj_plan_create.argtypes = [ctypes.POINTER(_lib.CmfView), ctypes.POINTER(P)]
    h.cmf_adj_plan_destroy.restype = None
    h.cmf_adj_plan_destroy.argtypes = [P]
    h.cmf_adj_sub_steps.restype = I
    h.cmf_adj_sub_steps.argtypes = [P, P, P, D, P]
    h.cmf_adj_forward.restype = I
    h.cmf_adj_forward.argtypes = [P, P, P, I, I, P, D]
    h.cmf_adj_reverse.restype = I
    h.cmf_adj_reverse.argtypes = [P, P, P, I, P, D, P, P, P, P]
    h.cmf_adj_finalize.restype = I
    h.cmf_adj_finalize.argtypes = [P, P, P, P, P]
    h._adj_bound = True


class AdjointRouting:
    """Gradient engine bound to a `CaMaFlood` model.

    The model must use precision "float64" and one member; its topology,
    fixed geometry and module tables are used, while the four differentiated
    parameters are passed per window.

    gauges            model-order indices of the cells whose discharge
                      (river + floodplain outflow at each interval end) the
                      window returns
    checkpoint_every  sub-steps between stored states (the recompute segment)
    """

    def __init__(self, model, gauges, checkpoint_every: int = 96):
        if model.precision != "float64":
            raise ValueError("the adjoint runs in fp64: build the model with precision='float64'")
        if model.num_members != 1:
            raise ValueError("the adjoint takes a single-member model")
        if checkpoint_every < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.model = model
        self.device = model.device
        self.N = model.num_catchments
        bm = model.bifurcation
        self.P = bm.num_bifurcation_paths if bm is not None else 0
        self.L = bm.num_bifurcation_levels if bm is not None else 0
        self.outer = model.step_seconds
        self.K = int(checkpoint_every)
        self.gauges = torch.as_tensor(gauges, dtype=torch.long, device=self.device)
        self.lib = _lib.lib()
        _bind(self.lib)
        b = model.base
        plan = self._plan(*(getattr(b, k).detach().contiguous() for k in PARAMS))
        try:
            sl, tl, sc = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
            gf = ctypes.c_int()
            _lib.check(self.lib.cmf_adj_sizes(plan, ctypes.byref(sl), ctypes.byref(tl),
                                              ctypes.byref(sc), ctypes.byref(gf)), "adj_sizes")
        finally:
            self.lib.cmf_adj_plan_destroy(plan)
        self.state_len, self.slot_len, self.scratch_len, self.n_grad = (
            sl.value, tl.value, sc.value, gf.value)
        assert self.state_len == len(CELL_STATE) * self.N + 2 * self.P * self.L
        assert self.n_grad == len(PARAMS)
        self._cells = len(CELL_STATE) * self.N
        self._path_off = SLOT_CELL_FIELDS * self.N
        self._n_dev = torch.zeros(1, dtype=torch.int32, device=self.device)

    # ------------------------------------------------------------------ #
    def pack(self, fields: dict) -> torch.Tensor:
        """Flat state from a dict of model-ordered tensors (missing module
        fields are zero)."""
        n, pl = self.N, self.P * self.L
        out = torch.zeros(self.state_len, dtype=torch.float64, device=self.device)
        for f, name in enumerate(CELL_STATE):
            if name in fields:
                out[f * n:(f + 1) * n] = fields[name].reshape(-1).to(out)
        for f, name in enumerate(PATH_STATE):
            if name in fields and pl:
                out[self._cells + f * pl:self._cells + (f + 1) * pl] = fields[name].reshape(-1).to(out)
        return out

    def unpack(self, state: torch.Tensor) -> dict:
        """Views of a flat state by field name ([N] cells, [P, L] paths)."""
        n, pl = self.N, self.P * self.L
        out = {name: state[f * n:(f + 1) * n] for f, name in enumerate(CELL_STATE)}
        if pl:
            for f, name in enumerate(PATH_STATE):
                out[name] = state[self._cells + f * pl:self._cells + (f + 1) * pl].view(self.P, self.L)
        return out

    def initial_state(self) -> torch.Tensor:
        """The model's current state as a flat fp64 tensor."""
        m = self.model
        fields = {k: getattr(m.base, k).detach() for k in CELL_STATE if hasattr(m.base, k)}
        if m.reservoir is not None:
            fields["reservoir_total_inflow"] = m.reservoir.reservoir_total_inflow.detach()
        if m.bifurcation is not None:
            for k in PATH_STATE:
                fields[k] = getattr(m.bifurcation, k).detach()
        return self.pack(fields)

    def parameters(self) -> dict[str, torch.Tensor]:
        """Copies of the model's four differentiable parameters."""
        b = self.model.base
        return {k: getattr(b, k).detach().clone() for k in PARAMS}

    def _plan(self, rman, fman, rh, rw):
        v = self.model._view()
        v.river_manning = rman.data_ptr()
        v.flood_manning = fman.data_ptr()
        v.river_height = rh.data_ptr()
        v.river_width = rw.data_ptr()
        plan = ctypes.c_void_p()
        _lib.check(self.lib.cmf_adj_plan_create(ctypes.byref(v), ctypes.byref(plan)),
                   "adj_plan_create")
        return plan

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _sub_steps(self, plan, slot: torch.Tensor) -> int:
        _lib.check(self.lib.cmf_adj_sub_steps(plan, self._stream(), slot.data_ptr(), self.outer,
                                              self._n_dev.data_ptr()), "adj_sub_steps")
        n = int(self._n_dev.item())
        if n < 1 or n > 100_000:
            raise FloatingPointError(f"CFL sub-step count {n} out of range (non-finite depth?)")
        return n

    # slot <-> state copies (the slot holds the state's cell fields first and
    # its path fields at the start of the path area)
    def _state_to_slot(self, state, slot):
        slot[:self._cells].copy_(state[:self._cells])
        pl2 = 2 * self.P * self.L
        if pl2:
            slot[self._path_off:self._path_off + pl2].copy_(state[self._cells:])

    def _slot_to_state(self, slot, state):
        state[:self._cells].copy_(slot[:self._cells])
        pl2 = 2 * self.P * self.L
        if pl2:
            state[self._cells:].copy_(slot[self._path_off:self._path_off + pl2])

    def window(self, params: dict, forcing: torch.Tensor, state0: torch.Tensor):
        """Differentiable window: returns (discharge [T, G], final flat state)."""
        return RoutingWindow.apply(self, params["river_manning"], params["flood_manning"],
                                   params["river_height"], params["river_width"], forcing, state0)

    @torch.no_grad()
    def forward_only(self, params: dict, forcing: torch.Tensor, state0: torch.Tensor):
        """The window's forward without checkpoints (for timing and FD checks)."""
        out = self._forward(params["river_manning"], params["flood_manning"],
                            params["river_height"], params["river_width"], forcing, state0,
                            keep_checkpoints=False)
        return out[0], out[1]

    # ------------------------------------------------------------------ #
    def _prep(self, *ts):
        return [t.detach().to(device=self.device, dtype=torch.float64).contiguous() for t in ts]

    def _forward(self, rman, fman, rh, rw, forcing, state0, keep_checkpoints=True):
        rman, fman, rh, rw, forcing, state0 = self._prep(rman, fman, rh, rw, forcing, state0)
        N = self.N
        if state0.numel() != self.state_len or forcing.dim() != 2 or forcing.shape[1] != N:
            raise ValueError("state0 must be the flat state and forcing [T, N], model order")
        state0 = state0.reshape(-1)
        plan = self._plan(rman, fman, rh, rw)
        try:
            slots = torch.zeros((2, self.slot_len), dtype=torch.float64, device=self.device)
            self._state_to_slot(state0, slots[0])
            cur = torch.empty_like(state0)
            stream = self._stream()
            T = forcing.shape[0]
            q = torch.empty((T, self.gauges.numel()), dtype=torch.float64, device=self.device)
            counts, ckpts, g = [], {}, 0
            for t in range(T):
                n = self._sub_steps(plan, slots[0])
                dt = self.outer / n
                k = 0
                while k < n:
                    if keep_checkpoints and g % self.K == 0:
                        self._slot_to_state(slots[0], cur)
                        ckpts[g] = cur.clone()
                    m = min(n - k, self.K - g % self.K)
                    _lib.check(self.lib.cmf_adj_forward(plan, stream, slots.data_ptr(), m, 0,
                                                        forcing[t].data_ptr(), dt), "adj_forward")
                    if m & 1:
                        slots[0].copy_(slots[1])
                    k += m
                    g += m
                counts.append(n)
                q[t] = (slots[0, F_ROUT * N:(F_ROUT + 1) * N]
                        + slots[0, F_FOUT * N:(F_FOUT + 1) * N])[self.gauges]
            final = torch.empty_like(state0)
            self._slot_to_state(slots[0], final)
        finally:
            self.lib.cmf_adj_plan_destroy(plan)
        return q, final, counts, ckpts, (rman, fman, rh, rw, forcing)

    def _backward(self, saved, counts, ckpts, q_bar, state_bar):
        rman, fman, rh, rw, forcing = saved
        N, dev = self.N, self.device
        T = forcing.shape[0]
        dts = [self.outer / n for n in counts]
        starts, ends, acc = [], [], 0
        for n in counts:
            starts.append(acc)
            acc += n
            ends.append(acc)
        total = acc
        lam = torch.zeros(self.state_len, dtype=torch.float64, device=dev)
        if state_bar is not None:
            lam += state_bar.reshape(-1).to(dev, torch.float64)
        lam_rout = lam[F_ROUT * N:(F_ROUT + 1) * N]
        lam_fout = lam[F_FOUT * N:(F_FOUT + 1) * N]
        grad = torch.zeros((self.n_grad, N), dtype=torch.float64, device=dev)
        g_forcing = torch.zeros((T, N), dtype=torch.float64, device=dev)
        scratch = torch.zeros(self.scratch_len, dtype=torch.float64, device=dev)
        seg_len = min(self.K, max(total, 1))
        # Two tapes: segment s-1 is recomputed on a side stream while segment s
        # is swept in reverse on the caller's stream (the two are independent).
        tapes = [torch.zeros((seg_len + 1, self.slot_len), dtype=torch.float64, device=dev)
                 for _ in range(2)]
        stride = self.slot_len * 8
        main = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(dev)
        side.wait_stream(main)
        for tp in tapes:
            tp.record_stream(side)
        ready = [torch.cuda.Event(), torch.cuda.Event()]
        free = [torch.cuda.Event(), torch.cuda.Event()]
        plan = self._plan(rman, fman, rh, rw)

        def recompute(s: int, buf: int):
            g0, g1 = s * self.K, min((s + 1) * self.K, total)
            tape = tapes[buf]
            chunks, g = [], g0
            with torch.cuda.stream(side):
                self._state_to_slot(ckpts[g0], tape[0])
                while g < g1:
                    t = bisect.bisect_right(starts, g) - 1
                    m = min(g1, ends[t]) - g
                    _lib.check(self.lib.cmf_adj_forward(
                        plan, side.cuda_stream, tape.data_ptr() + (g - g0) * stride, m, 1,
                        forcing[t].data_ptr(), dts[t]), "adj_forward(tape)")
                    chunks.append((t, g - g0, m))
                    g += m
            ready[buf].record(side)
            return g0, chunks

        try:
            n_seg = (total + self.K - 1) // self.K
            pending = recompute(n_seg - 1, 0) if n_seg else None
            for idx, s in enumerate(range(n_seg - 1, -1, -1)):
                buf = idx & 1
                g0, chunks = pending
                if s > 0:
                    if idx >= 1:
                        side.wait_event(free[1 - buf])
                    pending = recompute(s - 1, 1 - buf)
                main.wait_event(ready[buf])
                tape = tapes[buf]
                for t, j0, m in reversed(chunks):
                    if q_bar is not None and g0 + j0 + m == ends[t]:
                        qb = q_bar[t].to(dev, torch.float64)
                        lam_rout.index_add_(0, self.gauges, qb)
                        lam_fout.index_add_(0, self.gauges, qb)
                    _lib.check(self.lib.cmf_adj_reverse(
                        plan, main.cuda_stream, tape.data_ptr() + j0 * stride, m,
                        forcing[t].data_ptr(), dts[t], lam.data_ptr(), grad.data_ptr(),
                        g_forcing[t].data_ptr(), scratch.data_ptr()), "adj_reverse")
                free[buf].record(main)
            _lib.check(self.lib.cmf_adj_finalize(plan, main.cuda_stream, lam.data_ptr(),
                                                 grad.data_ptr(), scratch.data_ptr()),
                       "adj_finalize")
            main.wait_stream(side)
        finally:
            self.lib.cmf_adj_plan_destroy(plan)
        return grad, g_forcing, lam


class RoutingWindow(torch.autograd.Function):
    """(engine, river_manning, flood_manning, river_height, river_width,
    forcing [T, N], flat initial state) -> (discharge at the gauges [T, G],
    flat final state); all fp64, model order."""

    @staticmethod
    def forward(ctx, engine, rman, fman, rh, rw, forcing, state0):
        q, final, counts, ckpts, saved = engine._forward(rman, fman, rh, rw, forcing, state0)
        ctx.engine = engine
        ctx.counts = counts
        ctx.ckpts = ckpts
        ctx.saved = saved
        ctx.state_shape = state0.shape
        return q, final

    @staticmethod
    def backward(ctx, q_bar, state_bar):
        grad, g_forcing, lam = ctx.engine._backward(ctx.saved, ctx.counts, ctx.ckpts, q_bar,
                                                    state_bar)
        ctx.ckpts = None
        return None, grad[0], grad[1], grad[2], grad[3], g_forcing, lam.view(ctx.state_shape)
