"""Pure-PyTorch transcription of the reference sub-step -- TEST INFRASTRUCTURE.

The autograd reference of the hand-written adjoint (cmfb200.adjoint): tests run
a window through this transcription, take `torch.autograd.grad` of a loss and
compare with the CUDA reverse sweep, and check both against central finite
differences.  Only tests/ import it; the product never does.

It restates the base physics of one sub-step in the reference's step order
(cmfgpu/models/cama_flood_model.py:134-162):

  momentum   local-inertial river and floodplain flux, the opposite-flow
             rule and the negative-flow limiter       (cmfgpu/phys/cuda/outflow.cu:21-175)
  limiter    outgoing storage and limit rate            (outflow.cu:170-203)
  inflow     limited flux summed into the downstream cell  (outflow.cu:180-222)
  stage      fp64 storage update, flood stage over the floodplain table
                                                       (cmfgpu/phys/cuda/storage.cu:22-226)
  sub-steps  CFL count per forcing interval             (cmfgpu/phys/cuda/adaptive_time.cu:19-48)

Indices are whatever order the fields are given in (the physics is
index-based); the inflow scatter is an `index_add` over the downstream index,
mouths (downstream index == own index) excluded.

Subgradient convention, reproduced exactly by the hand-written adjoint:
  * `max(x, c)` / `min(x, c)` against a constant c are `clamp`: the gradient
    passes when x lies on or inside the bound;
  * `max(a, b)` of two varying operands is `torch.maximum`: at a tie each
    operand receives half;
  * a C ternary `cond ? a : b` is `where`: the gradient goes to the taken
    branch only;
  * `max(sqrt(p), f)` has gradient 1/(2 sqrt p) where p > f*f and 0
    elsewhere, so no `0 * inf` appears at p = 0;
  * |x| has gradient sign(x) (0 at 0); the flood level, the river/flood flow
    conditions and the CFL sub-step count are piecewise constant.
"""
from __future__ import annotations

import torch

STATE = ("river_storage", "flood_storage", "river_outflow", "flood_outflow", "river_depth",
         "flood_depth", "river_cross_section_depth", "flood_cross_section_depth",
         "flood_cross_section_area")
PARAMS = ("river_manning", "flood_manning", "river_height", "river_width")


def _sqrt_floor(p: torch.Tensor, floor: float) -> torch.Tensor:
    """max(sqrt(p), floor) with gradient 1/(2 sqrt p) for p > floor**2, else 0."""
    live = p > floor * floor
    return torch.where(live, torch.sqrt(torch.where(live, p, torch.ones_like(p))),
                       torch.full_like(p, floor))


def _cbrt(x: torch.Tensor) -> torch.Tensor:
    """Cube root of a positive tensor (the flow depths here are >= 1e-6)."""
    return x.pow(1.0 / 3.0)


class TorchRouting:
    """Base-physics sub-step in fp64 tensors.

    `fields` holds the static geometry in one consistent catchment order:
    downstream_idx, river_length, catchment_elevation, catchment_area,
    downstream_distance, flood_depth_table [N, K].  River height/width and
    the two Manning coefficients are passed per call (they are the
    differentiated parameters)."""

    def __init__(self, fields: dict, gravity: float = 9.8, adaptive_time_factor: float = 0.7,
                 max_sub_step_seconds: float = 0.0, device="cpu"):
        def t(name, dtype=torch.float64):
            return torch.as_tensor(fields[name]).to(device=device, dtype=dtype)

        self.dn = t("downstream_idx", torch.long)
        n = self.dn.shape[0]
        self.n = n
        self.mouth = self.dn == torch.arange(n, device=device)
        self.inner = ~self.mouth
        self.dn_inner = self.dn[self.inner]
        self.rl = t("river_length")
        self.celv = t("catchment_elevation")
        self.ca = t("catchment_area")
        self.dnd = t("downstream_distance")
        self.tbl = t("flood_depth_table")
        self.K = self.tbl.shape[1]
        self.g = float(gravity)
        self.alpha = float(adaptive_time_factor)
        self.max_dt = float(max_sub_step_seconds)

    # ------------------------------------------------------------------ #
    def sub_steps(self, s: dict, outer: float) -> int:
        """CFL count (adaptive_time.cu:19-48); piecewise constant, no gradient."""
        with torch.no_grad():
            depth = torch.clamp(s["river_depth"].detach(), min=0.01)
            dt = self.alpha * self.dnd / torch.sqrt(self.g * depth)
            if self.max_dt > 0:
                dt = torch.clamp(dt, max=self.max_dt)
            dt = torch.clamp(dt, max=outer)
            n = torch.floor(outer / dt - 0.01) + 1.0
            return int(n.max().item())

    def momentum(self, s: dict, p: dict, dt: float):
        """outflow.cu:21-175 (base physics)."""
        g = self.g
        mouth = self.mouth
        rh, rw = p["river_height"], p["river_width"]
        rman, fman = p["river_manning"], p["flood_manning"]
        rdep, fdep = s["river_depth"], s["flood_depth"]
        rout, fout = s["river_outflow"], s["flood_outflow"]
        rcsd, fcsd = s["river_cross_section_depth"], s["flood_cross_section_depth"]
        fcsa = s["flood_cross_section_area"]
        rs, fs = s["river_storage"], s["flood_storage"]
        celv, rl, dnd = self.celv, self.rl, self.dnd

        relev = celv - rh
        wse = rdep + relev
        wse_dn = torch.where(mouth, celv, rdep[self.dn] + relev[self.dn])
        max_wse = torch.maximum(wse, wse_dn)
        slope = (wse - wse_dn) / dnd
        fslope = torch.clamp(slope, -0.005, 0.005)

        ucsd = torch.where(mouth, rdep, max_wse - relev)
        r_sifd = _sqrt_floor(ucsd * rcsd, 1e-6)
        fsurf = torch.where(mouth, wse, max_wse)
        ufcsd = torch.clamp(fsurf - celv, min=0.0)
        f_sifd = _sqrt_floor(ufcsd * fcsd, 1e-6)
        ufcsa = torch.clamp(fs / rl - fdep * rw, min=0.0)

        river_cond = (r_sifd > 1e-5) & (ucsd * rw > 1e-5)
        q = rout / rw
        num = rw * (q + g * dt * r_sifd * slope)
        den = 1.0 + g * dt * (rman * rman) * torch.abs(q) * (1.0 / (r_sifd * r_sifd * _cbrt(r_sifd)))
        qr0 = torch.where(river_cond, num / den, torch.zeros_like(num))

        flood_cond = (f_sifd > 1e-5) & (ufcsa > 1e-5)
        f_imp = _sqrt_floor(ufcsa * torch.clamp(fcsa, min=1e-6), 1e-6)
        num_f = fout + g * dt * f_imp * fslope
        den_f = 1.0 + g * dt * (fman * fman) * torch.abs(fout) * (1.0 / (f_sifd * _cbrt(f_sifd))) / f_imp
        qf0 = torch.where(flood_cond, num_f / den_f, torch.zeros_like(num_f))

        qf1 = torch.where(qr0 * qf0 < 0.0, torch.zeros_like(qf0), qf0)
        neg = (qr0 < 0.0) & ~mouth
        total_neg = (-qr0 - qf1) * dt
        total_neg = torch.where(neg, total_neg, torch.ones_like(total_neg))
        lr_neg = torch.clamp(0.05 * (rs + fs) / total_neg, max=1.0)
        qr = torch.where(neg, qr0 * lr_neg, qr0)
        qf = torch.where(neg, qf1 * lr_neg, qf1)
        return qr, qf, ucsd, ufcsd, ufcsa

    def limit_rate(self, s: dict, qr, qf, dt: float):
        """Outgoing storage and limit rate (outflow.cu:170-174, :196-203)."""
        pos = torch.clamp(qr, min=0.0) + torch.clamp(qf, min=0.0)
        neg = torch.clamp(qr, max=0.0) + torch.clamp(qf, max=0.0)
        og = pos * dt
        og = og.index_add(0, self.dn_inner, -neg[self.inner] * dt)
        store = s["river_storage"] + s["flood_storage"]
        live = og > 1e-8
        ratio = store / torch.where(live, og, torch.ones_like(og))
        return torch.where(live, torch.clamp(ratio, max=1.0), torch.ones_like(og))

    def flood_stage(self, total, rh, rw):
        """storage.cu:118-211: river/flood split, depths and flooded fraction."""
        rl, ca, H, K = self.rl, self.ca, self.tbl, self.K
        rmax = rl * rw * rh
        flooded = total > rmax
        width_inc = (ca / rl) / K
        lv = torch.arange(K, device=H.device, dtype=torch.float64)
        W = rw[:, None] + (lv[None, :] + 1.0) * width_inc[:, None]
        W_prev = torch.cat([rw[:, None], W[:, :-1]], dim=1)
        H_prev = torch.cat([torch.zeros_like(H[:, :1]), H[:, :-1]], dim=1)
        dS = rl[:, None] * 0.5 * (W_prev + W) * (H - H_prev)
        S = rmax[:, None] + torch.cumsum(dS, dim=1)
        level = torch.cumprod((total[:, None] > S).to(torch.int64), dim=1).sum(dim=1)
        top = level == K
        lm1 = (level - 1).clamp(min=0)[:, None]
        S_prev = torch.where(level == 0, rmax, S.gather(1, lm1)[:, 0])
        D_prev = torch.where(level == 0, torch.zeros_like(rmax), H.gather(1, lm1)[:, 0])
        D_next = H.gather(1, level.clamp(max=K - 1)[:, None])[:, 0]
        W_tot = rw + level.to(torch.float64) * width_inc
        excess = total - S_prev
        # above the top layer
        fdep_top = D_prev + excess / (W_tot * rl)
        # inside layer `level`
        grad = (D_next - D_prev) / width_inc
        grad = torch.where(top, torch.ones_like(grad), grad)
        arg = W_tot * W_tot + 2.0 * excess / (grad * rl)
        arg = torch.where(top | ~flooded, torch.ones_like(arg), arg)
        diff_w = torch.sqrt(arg) - W_tot
        fdep_mid = D_prev + diff_w * grad
        fdep = torch.where(top, fdep_top, fdep_mid)
        cap = rmax + rl * rw * fdep
        river = torch.where(cap < total, cap, total)
        d = total - river
        flood = torch.where(d < 0.0, torch.zeros_like(d), d)
        ff_mid = torch.clamp((W_tot + diff_w - rw) * rl / ca, 0.0, 1.0)
        ffr = torch.where(top, torch.ones_like(ff_mid), ff_mid)
        zero = torch.zeros_like(total)
        rs = torch.where(flooded, river, total)
        fs = torch.where(flooded, flood, zero)
        rdep = rs / (rl * rw)
        fdep = torch.where(flooded, fdep, zero)
        ffr = torch.where(flooded, ffr, zero)
        return rs, fs, rdep, fdep, ffr

    def substep(self, s: dict, p: dict, runoff, dt: float):
        """One sub-step; returns (new state dict, flood_fraction)."""
        qr, qf, ucsd, ufcsd, ufcsa = self.momentum(s, p, dt)
        lr = self.limit_rate(s, qr, qf, dt)
        lr_dn = lr[self.dn]
        u_r = torch.where(qr >= 0.0, qr * lr, qr * lr_dn)
        u_f = torch.where(qf >= 0.0, qf * lr, qf * lr_dn)
        zero = torch.zeros_like(u_r)
        rin = zero.index_add(0, self.dn_inner, u_r[self.inner])
        fin = zero.index_add(0, self.dn_inner, u_f[self.inner])
        rs, fs = s["river_storage"], s["flood_storage"]
        river_su = rs + (rin - u_r) * dt
        flood_su = fs + torch.where(river_su < 0.0, river_su, zero) + (fin - u_f) * dt
        river_su = torch.where(river_su > 0.0, river_su, zero)
        tt = river_su + flood_su
        river_su = torch.where(flood_su < 0.0, torch.where(tt > 0.0, tt, zero), river_su)
        flood_su = torch.where(flood_su > 0.0, flood_su, zero)
        total = river_su + flood_su + runoff * dt
        total = torch.where(total > 0.0, total, zero)
        rs1, fs1, rdep1, fdep1, ffr = self.flood_stage(total, p["river_height"], p["river_width"])
        out = {"river_storage": rs1, "flood_storage": fs1, "river_outflow": u_r,
               "flood_outflow": u_f, "river_depth": rdep1, "flood_depth": fdep1,
               "river_cross_section_depth": ucsd, "flood_cross_section_depth": ufcsd,
               "flood_cross_section_area": ufcsa}
        return out, ffr

    def window(self, s0: dict, p: dict, forcing, outer: float, gauges):
        """Run len(forcing) intervals; return (discharge river+flood outflow at
        `gauges` after each interval [T, G], final state, sub-step counts)."""
        s = dict(s0)
        q, counts = [], []
        for t in range(forcing.shape[0]):
            n = self.sub_steps(s, outer)
            dt = outer / n
            for _ in range(n):
                s, _ = self.substep(s, p, forcing[t], dt)
            counts.append(n)
            q.append((s["river_outflow"] + s["flood_outflow"])[gauges])
        return torch.stack(q), s, counts


def relative_misfit_loss(q, q_obs):
    """Sum of squared relative discharge misfit."""
    return (((q - q_obs) / q_obs) ** 2).sum()

