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

and, with the matching modules, the dam-upstream kinematic flow
(outflow.cu:137-153), the reservoir release (reservoir.cu:18-94), the
bifurcation path flux and its inflow (bifurcation.cu:21-156, levee.cu:263-341)
and the levee re-partition (levee.cu:29-261).

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
The reservoir, dam, bifurcation and levee branches write every C
`fmax(a, b)` / `fmin(a, b)` as `where(a >= b, a, b)` / `where(a <= b, a, b)`:
the gradient follows the first operand on a tie (against a constant this is
the clamp rule above), and sqrt / cube root have gradient 0 at 0.
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


def _wmax(a, b):
    """C fmax(a, b); the first operand is taken on a tie."""
    return torch.where(a >= b, a, b)


def _wmin(a, b):
    """C fmin(a, b); the first operand is taken on a tie."""
    return torch.where(a <= b, a, b)


def _ssqrt(x: torch.Tensor) -> torch.Tensor:
    """sqrt of a non-negative tensor with gradient 0 at 0."""
    live = x > 0
    return torch.where(live, torch.sqrt(torch.where(live, x, torch.ones_like(x))),
                       torch.zeros_like(x))


def _scbrt(x: torch.Tensor) -> torch.Tensor:
    """Cube root of a non-negative tensor with gradient 0 at 0."""
    live = x > 0
    return torch.where(live, torch.where(live, x, torch.ones_like(x)).pow(1.0 / 3.0),
                       torch.zeros_like(x))


def state_names(modules) -> tuple:
    """State fields the transcription carries for these modules."""
    mods = set(modules)
    names = STATE + ("protected_storage", "protected_depth")
    if "reservoir" in mods:
        names += ("reservoir_total_inflow",)
    if "bifurcation" in mods:
        names += ("bifurcation_outflow", "bifurcation_cross_section_depth")
    return names


class TorchRouting:
    """One sub-step in fp64 tensors.

    `fields` holds the static inputs in one consistent catchment order (the
    names of oracle.reference_fields or of CaMaFlood.export_fields):
    downstream_idx, river_length, catchment_elevation, catchment_area,
    downstream_distance, flood_depth_table [N, K], plus the levee, reservoir
    and bifurcation tables of the open `modules`.  River height/width and the
    two Manning coefficients are passed per call (they are the differentiated
    parameters)."""

    def __init__(self, fields: dict, modules=("base",), gravity: float = 9.8,
                 adaptive_time_factor: float = 0.7, max_sub_step_seconds: float = 0.0,
                 min_kinematic_slope: float = 1e-5, device="cpu"):
        def t(name, dtype=torch.float64):
            return torch.as_tensor(fields[name]).to(device=device, dtype=dtype)

        mods = set(modules)
        self.modules = mods
        self.lev, self.res, self.bif = "levee" in mods, "reservoir" in mods, "bifurcation" in mods
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
        self.min_kin = float(min_kinematic_slope)
        zeros_b = torch.zeros(n, dtype=torch.bool, device=device)
        self.is_levee = zeros_b.clone()
        if self.lev:
            self.lci = t("levee_catchment_idx", torch.long)
            self.is_levee[self.lci] = True
            self.l_crown = t("levee_crown_height")
            self.l_frac = t("levee_fraction")
            self.l_base = t("levee_base_height")
        self.is_res, self.dam_up, self.dam_rel = zeros_b.clone(), zeros_b.clone(), zeros_b.clone()
        if self.res:
            self.rci = t("reservoir_catchment_idx", torch.long)
            self.is_res = t("is_reservoir", torch.bool)
            self.dam_up = t("is_dam_upstream", torch.bool)
            self.dam_rel = t("is_dam_related", torch.bool)
            for k in ("conservation_volume", "emergency_volume", "adjustment_volume",
                      "effective_normal_outflow", "adjustment_outflow", "flood_control_outflow"):
                setattr(self, "r_" + k, t(k))
            self.res_dn = self.is_res[self.dn] & self.inner
        if self.bif:
            self.bci = t("bifurcation_catchment_idx", torch.long)
            self.bdi = t("bifurcation_downstream_idx", torch.long)
            self.bman = t("bifurcation_manning")
            self.bwid = t("bifurcation_width")
            self.blen = t("bifurcation_length")
            self.belv = t("bifurcation_elevation")
            self.L = self.bwid.shape[1]
        self.names = state_names(mods)

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
            n = torch.where(self.dam_rel, torch.ones_like(n), n)
            return int(n.max().item())

    def momentum(self, s: dict, p: dict, dt: float):
        """outflow.cu:21-175 (with the dam-upstream kinematic flow) and
        reservoir.cu:18-94."""
        g = self.g
        mouth = self.mouth
        rh, rw = p["river_height"], p["river_width"]
        rman, fman = p["river_manning"], p["flood_manning"]
        rdep, fdep = s["river_depth"], s["flood_depth"]
        rout, fout = s["river_outflow"], s["flood_outflow"]
        rcsd, fcsd = s["river_cross_section_depth"], s["flood_cross_section_depth"]
        fcsa = s["flood_cross_section_area"]
        rs, fs = s["river_storage"], s["flood_storage"]
        ps = s.get("protected_storage", torch.zeros_like(rs))
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
        lr_neg = torch.clamp(0.05 * (rs + fs + ps) / total_neg, max=1.0)
        qr = torch.where(neg, qr0 * lr_neg, qr0)
        qf = torch.where(neg, qf1 * lr_neg, qf1)

        if self.res:
            qr, qf = self._dam_upstream(s, p, dt, qr, qf)
            qr, qf = self._reservoir(s, dt, qr, qf)
        return qr, qf, ucsd, ufcsd, ufcsa

    def _dam_upstream(self, s, p, dt, qr, qf):
        """Kinematic flow of the cells right upstream of a dam (outflow.cu:137-153)."""
        rman, fman, rw = p["river_manning"], p["flood_manning"], p["river_width"]
        rdep, fdep = s["river_depth"], s["flood_depth"]
        rs, fs = s["river_storage"], s["flood_storage"]
        bed = (self.celv - self.celv[self.dn]) / self.dnd
        bed = _wmax(bed, torch.full_like(bed, self.min_kin))
        vel_r = (1.0 / rman) * torch.sqrt(bed) * _scbrt(rdep * rdep)
        kin_r = rw * rdep * vel_r
        kin_r = _wmin(kin_r, rs / dt)
        kin_r = _wmax(kin_r, torch.zeros_like(kin_r))
        bed_f = _wmin(bed, torch.full_like(bed, 0.005))
        vel_f = (1.0 / fman) * torch.sqrt(bed_f) * _scbrt(fdep * fdep)
        area = fs / self.rl - fdep * rw
        area = _wmax(area, torch.zeros_like(area))
        kin_f = area * vel_f
        kin_f = _wmin(kin_f, fs / dt)
        kin_f = _wmax(kin_f, torch.zeros_like(kin_f))
        return torch.where(self.dam_up, kin_r, qr), torch.where(self.dam_up, kin_f, qf)

    def release(self, total, inflow, dt):
        """Reservoir release of total storage `total` under `inflow`
        (reservoir.cu:18-94), one value per reservoir."""
        cons, emerg = self.r_conservation_volume, self.r_emergency_volume
        adj, n_out = self.r_adjustment_volume, self.r_effective_normal_outflow
        a_out, fc_out = self.r_adjustment_outflow, self.r_flood_control_outflow
        one = torch.ones_like(total)
        b1 = total <= cons
        b2 = ~b1 & (total <= adj)
        b3 = ~b1 & ~b2 & (total <= emerg)
        ro1 = n_out * _ssqrt(total / cons)
        frac2 = torch.where(b2, (total - cons) / (adj - cons), one)
        ro2 = n_out + torch.exp(3.0 * torch.log(frac2)) * (a_out - n_out)
        frac3 = torch.where(b3, (total - adj) / (emerg - adj), one)
        tmp = a_out + torch.exp(0.1 * torch.log(frac3)) * (fc_out - a_out)
        flood = n_out + ((total - cons) / (emerg - cons)) * (inflow - n_out)
        ro3 = torch.where(inflow >= fc_out, _wmax(flood, tmp), tmp)
        ro4 = torch.where(inflow >= fc_out, inflow, fc_out)
        ro = torch.where(b1, ro1, torch.where(b2, ro2, torch.where(b3, ro3, ro4)))
        ro = _wmax(ro, torch.zeros_like(ro))
        return _wmin(ro, total / dt)

    def _reservoir(self, s, dt, qr, qf):
        ci = self.rci
        total = s["river_storage"][ci] + s["flood_storage"][ci]
        inflow = s["reservoir_total_inflow"][ci] + self._runoff[ci]
        ro = self.release(total, inflow, dt)
        return qr.index_put((ci,), ro), qf.index_put((ci,), torch.zeros_like(ro))

    def path_flux(self, s: dict, p: dict, dt: float):
        """Bifurcation level fluxes with the path limiter (bifurcation.cu:21-129,
        levee.cu:263-341): (limited level fluxes [P, L], limited path sum,
        new cross-section depths [P, L])."""
        g = self.g
        rs, fs = s["river_storage"], s["flood_storage"]
        ps = s["protected_storage"]
        wse = s["river_depth"] + (self.celv - p["river_height"])
        pwse = torch.where(self.is_levee, _wmin(self.celv + s["protected_depth"], wse), wse)
        tot = torch.where(self.is_res, rs + fs, rs + fs + ps)
        ci, di = self.bci, self.bdi
        wse_c, wse_d = wse[ci], wse[di]
        max_wse = _wmax(wse_c, wse_d)
        max_pwse = _wmax(pwse[ci], pwse[di])
        slope = (wse_c - wse_d) / self.blen
        slope = _wmin(_wmax(slope, torch.full_like(slope, -0.005)), torch.full_like(slope, 0.005))
        bout, bcsd = s["bifurcation_outflow"], s["bifurcation_cross_section_depth"]
        upd, csd_new = [], []
        sum_out = torch.zeros_like(slope)
        for lv in range(self.L):
            elv = self.belv[:, lv]
            zero = torch.zeros_like(elv)
            if self.lev:
                cur = max_wse if lv == 0 else max_pwse
                upd_csd = _wmax(cur - elv, zero)
                if lv == 0:
                    sifd = _ssqrt(upd_csd * bcsd[:, lv])
                    sifd = torch.where(sifd <= 0.0, upd_csd, sifd)
                else:
                    sifd = upd_csd
            else:
                upd_csd = _wmax(max_wse - elv, zero)
                sifd = _wmax(_ssqrt(upd_csd * bcsd[:, lv]), _ssqrt(upd_csd * 0.01))
            live = sifd > 1e-5
            sf = torch.where(live, sifd, torch.ones_like(sifd))
            man, w, o = self.bman[:, lv], self.bwid[:, lv], bout[:, lv]
            unit_o = o / w
            num = w * (unit_o + g * dt * sf * slope)
            den = 1.0 + g * dt * (man * man) * torch.abs(unit_o) * (1.0 / (sf * sf * _cbrt(sf)))
            u = torch.where(live, num / den, zero)
            sum_out = sum_out + u
            upd.append(u)
            csd_new.append(upd_csd)
        m = _wmin(tot[ci], tot[di])
        denom = torch.abs(sum_out) * dt
        has = denom > 0
        x = 0.05 * m / torch.where(has, denom, torch.ones_like(denom))
        lr_p = torch.where(has, _wmin(x, torch.ones_like(x)), torch.ones_like(x))
        bout_lim = torch.stack([u * lr_p for u in upd], dim=1)
        return bout_lim, sum_out * lr_p, torch.stack(csd_new, dim=1)

    def limit_rate(self, s: dict, qr, qf, dt: float, bsum=None):
        """Outgoing storage and limit rate (outflow.cu:170-174, :196-203,
        bifurcation.cu:125-128)."""
        pos = torch.clamp(qr, min=0.0) + torch.clamp(qf, min=0.0)
        neg = torch.clamp(qr, max=0.0) + torch.clamp(qf, max=0.0)
        og = pos * dt
        og = og.index_add(0, self.dn_inner, -neg[self.inner] * dt)
        if bsum is not None:
            z = torch.zeros_like(bsum)
            og = og.index_add(0, self.bci, _wmax(bsum, z) * dt)
            og = og.index_add(0, self.bdi, -_wmin(bsum, z) * dt)
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


    def levee_stage(self, rs0, fs0, rdep0, fdep0, ffr0, rw, rh):
        """Levee re-partition (levee.cu:29-261) of the levee cells after their
        flood stage; all arguments are gathered at the levee cells.  Returns
        (river, flood, protected storage, river, flood, protected depth,
        flooded fraction)."""
        ci = self.lci
        rl, ca, H, K = self.rl[ci], self.ca[ci], self.tbl[ci], self.K
        crown, frac, base = self.l_crown, self.l_frac, self.l_base
        total = rs0 + fs0
        rmax = rl * rw * rh
        active = total >= rmax
        dwth_inc = (ca / rl) / K
        levee_dist = frac * (ca / rl)
        s_curr, dhgt_pre, dwth_pre = rmax, torch.zeros_like(rmax), rw
        base_sto, fill_sto = rmax, rmax
        f_base = torch.zeros_like(active)
        f_fill = torch.zeros_like(active)
        f_B = torch.zeros_like(active)
        ilev = (frac * K).to(torch.long)
        fil_B, wth_B, dph_B, grad_B = (torch.zeros_like(rmax) for _ in range(4))
        scan = torch.ones_like(active)
        tiny = torch.full_like(rmax, 1e-6)
        for l in range(K):
            depth_val = H[:, l]
            dhgt_seg = _wmax(depth_val - dhgt_pre, tiny)
            dwth_mid = dwth_pre + 0.5 * dwth_inc
            s_next = s_curr + rl * dwth_mid * dhgt_seg
            gradient = dhgt_seg / dwth_inc
            c_base = (base > dhgt_pre) & (base <= depth_val)
            r_base = (base - dhgt_pre) / dhgt_seg
            p_base = rl * (dwth_pre + 0.5 * r_base * dwth_inc) * (r_base * dhgt_seg)
            base_sto = torch.where(scan & c_base & ~f_base, s_curr + p_base, base_sto)
            f_base = torch.where(scan, f_base | c_base, f_base)
            c_fill = (crown > dhgt_pre) & (crown <= depth_val)
            r_fill = (crown - dhgt_pre) / dhgt_seg
            p_fill = rl * (dwth_pre + 0.5 * r_fill * dwth_inc) * (r_fill * dhgt_seg)
            fill_sto = torch.where(scan & c_fill & ~f_fill, s_curr + p_fill, fill_sto)
            f_fill = torch.where(scan, f_fill | c_fill, f_fill)
            s_top_loop = base_sto + (levee_dist + rw) * (crown - base) * rl
            threshold = s_next + (levee_dist + rw) * (crown - depth_val) * rl
            check = (ilev <= l) & ~f_B
            found = check & (total < threshold)
            current_lb = torch.where(ilev == l, s_top_loop, fil_B)
            a = check & ~found
            fil_B = torch.where(scan, torch.where(a, threshold, current_lb), fil_B)
            wth_B = torch.where(scan & a, dwth_inc * (l + 1) - levee_dist, wth_B)
            dph_B = torch.where(scan & a, depth_val - base, dph_B)
            grad_B = torch.where(scan & found, gradient, grad_B)
            f_B = torch.where(scan, f_B | found, f_B)
            s_curr = torch.where(scan, s_next, s_curr)
            dhgt_pre = torch.where(scan, depth_val, dhgt_pre)
            dwth_pre = torch.where(scan, dwth_pre + dwth_inc, dwth_pre)
            scan = scan & ~(f_base & f_fill & f_B)
        base_extra = s_curr + rl * dwth_pre * (base - dhgt_pre)
        base_sto = torch.where(f_base, base_sto, torch.where(base > dhgt_pre, base_extra, rmax))
        fill_extra = s_curr + rl * dwth_pre * (crown - dhgt_pre)
        fill_sto = torch.where(f_fill, fill_sto, torch.where(crown > dhgt_pre, fill_extra, rmax))
        s_top = base_sto + (levee_dist + rw) * (crown - base) * rl
        c4 = total >= fill_sto
        c3 = ~c4 & (total >= s_top)
        c2 = ~c4 & ~c3 & (total >= base_sto)
        zero = torch.zeros_like(total)
        f_dph_c2 = base + (total - base_sto) / (levee_dist + rw) / rl
        r_sto_c2 = rmax + rl * rw * f_dph_c2
        r_dph_c2 = r_sto_c2 / rl / rw
        f_sto_c2 = _wmax(total - r_sto_c2, zero)
        add_B = total - fil_B
        term_B = wth_B * wth_B + 2.0 * add_B / rl / (grad_B + 1e-9)
        p_dph_B = torch.where(f_B, base + dph_B + (-wth_B + _ssqrt(_wmax(term_B, zero))) * grad_B,
                              base + dph_B + add_B / (wth_B * rl + 1e-9))
        f_frc_B = torch.where(f_B, (wth_B + levee_dist) / (dwth_inc * K), torch.ones_like(total))
        r_sto_c3 = rmax + rl * rw * crown
        r_dph_c3 = r_sto_c3 / rl / rw
        f_sto_c3 = _wmax(s_top - r_sto_c3, zero)
        f_sto_c4 = _wmax(s_top + (fdep0 - crown) * (levee_dist + rw) * rl - rs0, zero)
        r_cand = torch.where(c2, r_sto_c2, torch.where(c3, r_sto_c3, torch.where(c4, rs0, rs0)))
        f_cand = torch.where(c2, f_sto_c2, torch.where(c3, f_sto_c3, torch.where(c4, f_sto_c4, fs0)))
        nolev = ~c2 & ~c3 & ~c4
        r_sto = torch.where(c4 | nolev, rs0, _wmin(r_cand, total))
        rem = total - r_sto
        rem = torch.where(rem > 0.0, rem, zero)
        f_sto = _wmin(torch.where(f_cand > 0.0, f_cand, zero), rem)
        f_sto = torch.where(c2, rem, f_sto)
        f_sto = torch.where(nolev, fs0, f_sto)
        p_sto = rem - f_sto
        p_sto = torch.where(p_sto > 0.0, p_sto, zero)
        r_dph = torch.where(c2, r_dph_c2, torch.where(c3, r_dph_c3, rdep0))
        f_dph = torch.where(c2, f_dph_c2, torch.where(c3, torch.zeros_like(total) + crown, fdep0))
        p_dph = torch.where(c2, zero, torch.where(c3, p_dph_B, torch.where(c4, fdep0, zero)))
        f_frc = torch.where(c2, frac + zero, torch.where(c3, torch.clamp(f_frc_B, 0.0, 1.0), ffr0))
        return (torch.where(active, r_sto, rs0), torch.where(active, f_sto, fs0),
                torch.where(active, p_sto, zero), torch.where(active, r_dph, rdep0),
                torch.where(active, f_dph, fdep0), torch.where(active, p_dph, zero),
                torch.where(active, f_frc, ffr0))

    def substep(self, s: dict, p: dict, runoff, dt: float):
        """One sub-step in the reference phase order; returns (new state dict,
        flood_fraction)."""
        self._runoff = runoff
        qr, qf, ucsd, ufcsd, ufcsa = self.momentum(s, p, dt)
        bsum = None
        if self.bif:
            bout_lim, bsum, bcsd_new = self.path_flux(s, p, dt)
        lr = self.limit_rate(s, qr, qf, dt, bsum)
        lr_dn = lr[self.dn]
        u_r = torch.where(qr >= 0.0, qr * lr, qr * lr_dn)
        u_f = torch.where(qf >= 0.0, qf * lr, qf * lr_dn)
        zero = torch.zeros_like(u_r)
        rin = zero.index_add(0, self.dn_inner, u_r[self.inner])
        fin = zero.index_add(0, self.dn_inner, u_f[self.inner])
        out = {}
        if self.res:
            mask = self.res_dn
            out["reservoir_total_inflow"] = zero.index_add(0, self.dn[mask], (u_r + u_f)[mask])
        gb = zero
        if self.bif:
            lr_c, lr_d = lr[self.bci], lr[self.bdi]
            out["bifurcation_outflow"] = torch.where(bout_lim >= 0.0, bout_lim * lr_c[:, None],
                                                     bout_lim * lr_d[:, None])
            out["bifurcation_cross_section_depth"] = bcsd_new
            raw = bout_lim[:, 0]
            for lv in range(1, self.L):
                raw = raw + bout_lim[:, lv]
            net = torch.where(raw >= 0.0, raw * lr_c, raw * lr_d)
            gb = zero.index_add(0, self.bci, net).index_add(0, self.bdi, -net)
        rs, fs = s["river_storage"], s["flood_storage"]
        prot = s.get("protected_storage", zero)
        river_su = rs + (rin - u_r) * dt
        flood_su = fs + torch.where(river_su < 0.0, river_su, zero) + (fin - u_f - gb) * dt
        river_su = torch.where(river_su > 0.0, river_su, zero)
        tt = river_su + flood_su
        river_su = torch.where(flood_su < 0.0, torch.where(tt > 0.0, tt, zero), river_su)
        flood_su = torch.where(flood_su > 0.0, flood_su, zero)
        total = river_su + flood_su + prot + runoff * dt
        total = torch.where(total > 0.0, total, zero)
        rs1, fs1, rdep1, fdep1, ffr = self.flood_stage(total, p["river_height"], p["river_width"])
        ps1, pdep1 = zero, fdep1
        if self.lev:
            ci = self.lci
            lv = self.levee_stage(rs1[ci], fs1[ci], rdep1[ci], fdep1[ci], ffr[ci],
                                  p["river_width"][ci], p["river_height"][ci])
            rs1, fs1, ps1 = rs1.index_put((ci,), lv[0]), fs1.index_put((ci,), lv[1]), ps1.index_put((ci,), lv[2])
            rdep1, fdep1 = rdep1.index_put((ci,), lv[3]), fdep1.index_put((ci,), lv[4])
            pdep1, ffr = pdep1.index_put((ci,), lv[5]), ffr.index_put((ci,), lv[6])
        out.update({"river_storage": rs1, "flood_storage": fs1, "river_outflow": u_r,
                    "flood_outflow": u_f, "river_depth": rdep1, "flood_depth": fdep1,
                    "river_cross_section_depth": ucsd, "flood_cross_section_depth": ufcsd,
                    "flood_cross_section_area": ufcsa, "protected_storage": ps1,
                    "protected_depth": pdep1})
        return out, ffr

    def window(self, s0: dict, p: dict, forcing, outer: float, gauges):
        """Run len(forcing) intervals; return (discharge river+flood outflow at
        `gauges` after each interval [T, G], final state, sub-step counts)."""
        s = dict(s0)
        s.setdefault("protected_storage", torch.zeros_like(s["river_storage"]))
        s.setdefault("protected_depth", torch.zeros_like(s["river_storage"]))
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

