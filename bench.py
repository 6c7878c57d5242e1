"""Benchmark: catchment-sub-steps/s of the CaMa-Flood routing path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload full_6m|full_250k|plain_60k]

A step is one forcing interval (`CaMaFlood.step_advance`, hourly for the
default 6M-catchment full-physics workload): the CFL sub-step count, then n
sub-steps of momentum -> limiter/inflow/stage, all in one CUDA graph launch.

Printed JSON (rank 0, one line):
  value       catchment-sub-steps/s with forcing already resident in HBM
              (sum over ranks of N x sub-steps, / max-over-ranks device time)
  e2e         the same metric through the public API with host buffers: every
              step copies its runoff from pinned host memory and reads gauge
              discharge back to the host, both inside the timed region
  roofline    algorithmic bytes of one sub-step (momentum + stage kernels),
              timed per kernel with CUDA events on the launch stream, against
              the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle port timed on this host's cores (bounded sample)

`--impl reference` times the reference algorithm's CPU restatement (the oracle
port: the reference ships no CPU path) on all host cores for the same workload.
Multi-GPU (torchrun): every rank routes its own set of basins (an independent
network of the same size; weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "cama-flood-gpu_b200"))

METRIC = "catchment-substeps/s: fwd, fwd+adjoint, 64-member batch vs plain, same GPU"
UNIT = "catchment-substeps/s"


def algorithmic_bytes(n: int, n_paths: int, n_levees: int, n_res: int, full: bool) -> float:
    """Compulsory bytes of one sub-step: every parameter read once, every state
    read and written once, forcing read once (no intermediates).
    Per catchment: parameters 76 (9 fp32 + 40 B flood table) + runoff 4 +
    state read 44 + state write 48 = 172.  Full physics adds per catchment
    protected storage (16 r+w) + protected depth (8 r+w) + levee/dam masks (3),
    16 per levee (index, crown, fraction, base), 152 per bifurcation path
    (12 + 5 levels x (12 read + 16 read/write)) and 44 per reservoir."""
    b = 172.0 * n
    if full:
        b += 27.0 * n + 16.0 * n_levees + 152.0 * n_paths + 44.0 * n_res
    return b


def fp64_algorithmic_bytes(n: int, n_paths: int, n_levees: int, n_res: int) -> float:
    """The full-physics rule of algorithmic_bytes with every REAL field in fp64
    (the adjoint's primal): per catchment the downstream index 4 + 8 parameters
    x 8 + flood table 80 + runoff 8 + state read 72 + state write 80 = 308, plus
    protected storage 16 + protected depth 16 + masks 3; 28 per levee; per
    bifurcation path 8 + 8 + 5 levels x (24 read + 32 read/write) = 296; 72 per
    reservoir."""
    return 343.0 * n + 28.0 * n_levees + 296.0 * n_paths + 72.0 * n_res


def adjoint_algorithmic_bytes(n: int, n_paths: int, n_levees: int, n_res: int, state_len: int,
                              slot_len: int, n_grad: int) -> float:
    """Compulsory bytes of one sub-step of forward+adjoint with checkpoints:
    the primal twice (the checkpointed forward and the taped recompute), the
    tape slot written once and read once, the parameters read by the reverse
    sweep (fp64: 148 per catchment, 28 per levee, 136 per path, 56 per
    reservoir), the adjoint state read and written (state_len doubles), and
    n_grad per-catchment parameter gradients accumulated (read and write)."""
    fwd = fp64_algorithmic_bytes(n, n_paths, n_levees, n_res)
    params = 148.0 * n + 28.0 * n_levees + 136.0 * n_paths + 56.0 * n_res
    return (2.0 * fwd + 2.0 * 8.0 * slot_len + params + 2.0 * 8.0 * state_len
            + 16.0 * n_grad * n)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(gpu_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def build_workload(name: str, seed_offset: int, topo=None):
    """The seeded network of workload `name`; `topo` replaces the product's
    integration helpers (the reference arm passes the oracle's, so that it
    never loads libcmfb200)."""
    from cmfb200 import synthetic as syn
    cfg = dict(syn.CONFIGS[name])
    spec = cfg["spec"]
    spec = syn.NetworkSpec(**{**spec.__dict__, "seed": spec.seed + seed_offset})
    net = syn.generate(spec, topo=topo)
    return net, cfg


def intervals_per_day(cfg) -> int:
    return max(1, int(round(86400.0 / cfg["interval"])))


def runoff_series(net, cfg, count: int, start: int = 0) -> np.ndarray:
    """Forcing of intervals start .. start+count-1 (input order), float32 m^3/s:
    daily gamma runoff, split by a random diurnal profile for sub-daily
    intervals."""
    from cmfb200 import synthetic as syn
    out = np.empty((count, net.num_catchments), dtype=np.float32)
    if cfg["interval"] >= 86400.0:
        for j in range(count):
            out[j] = syn.daily_runoff(net, start + j)
    else:
        per_day = intervals_per_day(cfg)
        day = None
        for j in range(count):
            d, h = divmod(start + j, per_day)
            if d != day:
                daily = syn.daily_runoff(net, d)
                prof = syn.diurnal_profile(d, seed=net.spec.seed, hours=per_day)
                day = d
            out[j] = daily * prof[h]
    return out


def spin_up(net, cfg, days: int, device, order, set_runoff, advance) -> int:
    """Route `days` simulated days (the first days*intervals_per_day intervals
    of runoff_series, same values) before anything is timed, so that timing
    sees a flooded, spun-up state instead of the cold start.  Daily runoff is
    uploaded once per day and split on the device (float32 products, equal to
    runoff_series').  `order` maps the caller's catchment order to input
    order (None: input order).  Returns the intervals routed."""
    import torch
    from cmfb200 import synthetic as syn
    per_day = intervals_per_day(cfg)
    for d in range(days):
        daily = syn.daily_runoff(net, d)
        if order is not None:
            daily = daily[order]
        dev = torch.as_tensor(daily).to(device)
        if cfg["interval"] >= 86400.0:
            set_runoff(dev)
            advance()
            continue
        prof = syn.diurnal_profile(d, seed=net.spec.seed, hours=per_day)
        for h in range(per_day):
            set_runoff(dev * float(prof[h]))
            advance()
    return days * (per_day if cfg["interval"] < 86400.0 else 1)


def workload_config(args, net, cfg, world: int) -> dict:
    """The `config` object of both arms (identical keys and values)."""
    f = net.fields
    return {"workload": args.workload, "catchments_per_gpu": net.num_catchments,
            "bifurcation_paths": int(f["bifurcation_catchment_id"].shape[0])
            if "bifurcation_catchment_id" in f else 0,
            "levees": int(f["levee_catchment_id"].shape[0]) if "levee_catchment_id" in f else 0,
            "reservoirs": int(f["reservoir_catchment_id"].shape[0])
            if "reservoir_catchment_id" in f else 0,
            "interval_s": cfg["interval"], "spinup_days": args.spinup_days,
            "parallelism": f"basin-sharded x{world}" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (state ~1 GB)"}


def loaded_native_libraries() -> list[str]:
    """In-tree shared libraries mapped into this process."""
    seen = []
    try:
        with open("/proc/self/maps") as fh:
            for line in fh:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and str(ROOT) in path and path not in seen:
                    seen.append(path)
    except OSError:
        pass
    return [str(Path(p).relative_to(ROOT)) if p.startswith(str(ROOT)) else p for p in seen]


def cpu_sample(net, cfg, model_dt_hint: float | None, target_seconds: float = 15.0):
    """Time the CPU oracle port (all host threads) on a bounded sample."""
    from oracle import oracle as O
    fields = O.reference_fields(net.fields, net.opened_modules)
    orc = O.Oracle(fields, net.opened_modules)
    threads = O.max_threads()
    from cmfb200 import synthetic as syn
    orc.set_runoff(runoff_series(net, cfg, 1)[0])
    n = orc.adaptive_sub_steps(cfg["interval"], cfg.get("max_sub_step_seconds", 0.0))
    orc.set_time_step(cfg["interval"] / max(n, 1), cfg["interval"])
    t0 = time.perf_counter()
    orc.substep()
    one = time.perf_counter() - t0
    reps = max(1, min(200, int(target_seconds / max(one, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(reps):
        orc.substep()
    dt = time.perf_counter() - t0
    # the same port on one core, a shorter sample (about a third of the time)
    O.set_threads(1)
    try:
        t0 = time.perf_counter()
        orc.substep()
        one1 = time.perf_counter() - t0
        reps1 = max(1, min(200, int(target_seconds / 3.0 / max(one1, 1e-6))))
        t0 = time.perf_counter()
        for _ in range(reps1):
            orc.substep()
        dt1 = time.perf_counter() - t0
    finally:
        O.set_threads(threads)
    return {
        "value": net.num_catchments * reps / dt,
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"{reps} sub-steps of the {net.num_catchments}-catchment network "
                  f"(oracle/cmf_oracle.c, OpenMP, {threads} threads), dt={cfg['interval'] / max(n, 1):.1f}s",
        "value_1_core": net.num_catchments * reps1 / dt1,
        "sample_1_core": f"{reps1} sub-steps, 1 thread",
    }


def forcing_measure(device, net, desired_ids, steps: int = 24, grid_shape=(720, 1440),
                    repeats: int = 10) -> dict:
    """The forcing map in front of the path: a chunk of `steps` gridded runoff
    fields (0.25-degree global grid, float32 mm/day) mapped onto the
    workload's catchments (model order) by cmf_forcing_apply.  Kernel time by
    CUDA events with the chunk resident; chunk e2e adds the pinned-host H2D
    copy of the chunk; the CPU restatement (oracle scipy product) is timed
    on one series and scaled."""
    import torch
    from cmfb200 import synthetic as syn
    from cmfb200.forcing import apply_mapping, build_local_mapping, local_csr
    from oracle import forcing as OF
    tab = syn.runoff_mapping(net, grid_shape, seed=7)
    m = build_local_mapping(tab, desired_ids, device)
    chunk = torch.from_numpy(syn.gridded_runoff(grid_shape, steps, seed=3)).pin_memory()
    dev = chunk.to(device)
    out = torch.empty((steps, m.num_rows), dtype=torch.float32, device=device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)     # > L2
    stream = torch.cuda.current_stream(device)
    for _ in range(3):
        apply_mapping(m, dev, out=out, unit_factor=86400000.0)
    times = []
    for _ in range(repeats):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        apply_mapping(m, dev, out=out, unit_factor=86400000.0)
        b.record(stream)
        torch.cuda.synchronize(device)
        times.append(a.elapsed_time(b))
    ms = float(np.mean(times))
    e2e = []
    for _ in range(repeats):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dev.copy_(chunk, non_blocking=True)
        apply_mapping(m, dev, out=out, unit_factor=86400000.0)
        b.record(stream)
        torch.cuda.synchronize(device)
        e2e.append(a.elapsed_time(b))
    alg = m.bytes_per_launch(steps, 4, 4)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    rp, col, w, G = local_csr(tab, desired_ids)
    g1 = chunk[0].numpy().reshape(1, -1).astype(np.float64)
    t0 = time.perf_counter()
    OF.scipy_map(rp, col, w, g1, G)
    cpu_one = time.perf_counter() - t0
    return {
        "workload": f"{m.num_rows} catchments x {steps} steps, grid {grid_shape[0]}x{grid_shape[1]}, "
                    f"nnz {m.nnz}",
        "ms_per_chunk": ms, "ms_per_chunk_e2e": float(np.mean(e2e)),
        "h2d_bytes_per_chunk": int(chunk.numel() * 4),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": alg, "kernel": "k_forcing_map"},
        "cpu_ms_per_chunk": cpu_one * steps * 1e3,
        "cpu_sample": "one step of the chunk through scipy.sparse CSR (1 thread), x steps",
    }


def statistics_overhead(model, dev_forcing, first: int, steps: int, base_ms: float,
                        base_substeps: int) -> dict:
    """The reference run scripts' output statistics ({"mean": total_outflow,
    "last": river_depth}) accumulated in the interval graph: the same timed
    intervals with and without them."""
    import torch
    spec = {"mean": ["total_outflow"], "last": ["river_depth"]}
    model.set_variables_to_save(spec)
    device = model.device
    for k in range(2):
        model.set_inputs(dev_forcing[first + k])
        model.step_advance()
    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    counts = torch.zeros(steps, dtype=torch.int32, device=device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for j, k in enumerate(range(first, first + steps)):
        model.set_inputs(dev_forcing[k])
        model.step_advance()
        counts[j].copy_(model.sub_step_counts()[0])
    b.record(stream)
    torch.cuda.synchronize(device)
    ms = a.elapsed_time(b)
    sub = int(counts.sum().item())
    stats = model.collect_statistics()
    ok = all(bool(torch.isfinite(v).all()) for v in stats.values())
    model.set_variables_to_save(None)
    with_ms = ms / max(sub, 1)
    without_ms = base_ms / max(base_substeps, 1)
    return {"variables_to_save": spec, "ms_per_substep": with_ms,
            "ms_per_substep_without": without_ms, "overhead_frac": with_ms / without_ms - 1.0,
            "sub_steps": sub, "finite": ok}


ENSEMBLE_CHECK_FIELDS = ("river_storage", "flood_storage", "river_outflow", "flood_outflow",
                         "river_depth", "flood_depth", "flood_fraction")


def _bit_sums(t):
    """Sum over catchments of the integer bit patterns of a state field
    ([N] -> scalar, [N, M] -> [M]): equal states give equal sums, and a single
    differing bit changes them."""
    import torch
    as_int = t.contiguous().view(torch.int64 if t.element_size() == 8 else torch.int32)
    return as_int.to(torch.int64).sum(dim=0)


def ensemble_compare(device, members: int, catchments: int, basins: int = 500,
                     member_tile: int = 16, block: int = 64, days: int = 5) -> dict:
    """The batched-ensemble workload: `members` members of a `basins`-basin
    network (~`catchments` catchments per member, 6M by default; runoff and
    river Manning perturbed per member, daily forcing, per-member dt).  The
    first `days` simulated days of the 30-day window (a bounded sample) in a
    single member-innermost model (one launch per phase) against the same
    members run one after another as plain models over the same days, both
    from the same initial state on the same GPU.  The batched model runs
    `member_tile` members of a catchment per thread in CTAs of `block` threads
    (member_tile 0: the autotuner picks both on the first day); the looped
    plain models keep their default CTA size.  Forcing of every day and member
    is resident on the device before timing.  Each member's end state is
    checked against its looped run (bit-pattern sums of seven state fields;
    the looped fingerprints are timed apart and left out of the looped time)."""
    import torch
    from cmfb200 import CaMaFlood, synthetic as syn
    net = syn.generate_basins(basins, catchments, seed=3)
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=3)
    manning = (net.fields["river_manning"][:, None] * mfac).astype(np.float32)
    mods = ["base", "adaptive_time"]
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods,
                    num_members=members, batched_fields={"river_manning": manning},
                    **({"BLOCK_SIZE": block} if member_tile > 0 else {}))
    order = ens.order
    rfac_dev = torch.as_tensor(np.ascontiguousarray(rfac[order])).to(device)
    daily = torch.stack([torch.as_tensor(syn.daily_runoff(net, d)[order]) for d in range(days)]).to(device)
    forcing = daily[:, :, None] * rfac_dev[None]               # [D, N, M] float32
    init = {k: v.clone() for k, v in ens.state_tensors().items()}
    stream = torch.cuda.current_stream(device)

    def reset(model, state):
        for k, v in model.state_tensors().items():
            v.copy_(state[k])

    ens.set_inputs(forcing[0])
    if member_tile > 0:
        ens.set_member_tile(member_tile)
    else:
        ens.autotune_block_size(sub_steps=2)
    ens.step_advance()                      # builds the interval graph
    reset(ens, init)
    torch.cuda.synchronize(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cnt_b = torch.zeros((days, members), dtype=torch.int32, device=device)
    a.record(stream)
    for d in range(days):
        ens.set_inputs(forcing[d])
        ens.step_advance()
        cnt_b[d].copy_(ens.sub_step_counts())
    b.record(stream)
    torch.cuda.synchronize(device)
    t_batched = a.elapsed_time(b) / 1e3
    n_batched = int(cnt_b.sum().item())
    tile, block = ens.member_tile, ens.block_size
    # each member's end state, as integer sums of the bit patterns of its fields
    fp_b = torch.stack([_bit_sums(getattr(ens.base, k)) for k in ENSEMBLE_CHECK_FIELDS])  # [F, M]
    ens.close()
    del ens, init, forcing

    plain = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=mods)
    init = {k: v.clone() for k, v in plain.state_tensors().items()}
    man_dev = torch.as_tensor(np.ascontiguousarray(manning[order].T)).to(device)
    run_dev = (daily[None, :, :] * rfac_dev.T[:, None, :]).contiguous()   # [M, D, N]
    plain.base.river_manning.copy_(man_dev[0])
    plain.set_inputs(run_dev[0, 0])
    plain.step_advance()                    # graph build
    torch.cuda.synchronize(device)
    a.record(stream)
    cnt_l = torch.zeros((members, days), dtype=torch.int32, device=device)
    fp_l = torch.zeros((len(ENSEMBLE_CHECK_FIELDS), members), dtype=torch.int64, device=device)
    f_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(members)]
    for m in range(members):
        reset(plain, init)
        plain.base.river_manning.copy_(man_dev[m])
        for d in range(days):
            plain.set_inputs(run_dev[m, d])
            plain.step_advance()
            cnt_l[m, d].copy_(plain.sub_step_counts()[0])
        f_ev[m][0].record(stream)
        for j, k in enumerate(ENSEMBLE_CHECK_FIELDS):
            fp_l[j, m] = _bit_sums(getattr(plain.base, k))
        f_ev[m][1].record(stream)
    b.record(stream)
    torch.cuda.synchronize(device)
    # the end-state fingerprints are not part of the looped runs' time
    t_looped = (a.elapsed_time(b) - sum(e0.elapsed_time(e1) for e0, e1 in f_ev)) / 1e3
    state_equal = bool(torch.equal(fp_b, fp_l))
    n_looped = int(cnt_l.sum().item())
    same_counts = bool(torch.equal(cnt_b, cnt_l.T))
    plain.close()
    del run_dev, daily, rfac_dev
    torch.cuda.empty_cache()
    batched = n * n_batched / t_batched
    looped = n * n_looped / t_looped
    # algorithmic bytes (plain physics): a looped cell-sub-step moves the
    # 172 B of algorithmic_bytes; a batched member-cell-sub-step moves its own
    # state, runoff and river Manning (44 + 48 + 4 + 4 = 100 B) and a 1/M
    # share of the other, shared parameters (72 B)
    b_batched = 100.0 + 72.0 / members
    b_looped = algorithmic_bytes(1, 0, 0, 0, False)
    peak, peak_kind = measured_peak()
    roof = {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_kind": peak_kind,
            "batched_bytes_per_member_substep": b_batched, "looped_bytes_per_substep": b_looped,
            "batched_achieved": b_batched * batched / 1e9,
            "batched_frac": b_batched * batched / 1e9 / peak,
            "looped_achieved": b_looped * looped / 1e9, "looped_frac": b_looped * looped / 1e9 / peak}
    return {"value": batched, "looped_value": looped, "speedup": batched / looped, "roofline": roof,
            "unit": UNIT, "members": members, "catchments_per_member": n, "basins": basins,
            "member_tile": tile, "block": block, "days": days,
            "sub_steps_per_member_mean": n_batched / members,
            "same_sub_step_counts": same_counts,
            "members_equal_looped_runs": state_equal,
            "checked_fields": list(ENSEMBLE_CHECK_FIELDS),
            "workload": f"{days} days (a sample of the 30-day window) of a member-innermost "
                        "ensemble (runoff x lognormal(0.3), river Manning x U(0.8,1.2) per member) "
                        "vs the members looped as plain models over the same days; includes the "
                        "state reset copies of the looped runs"}


def small_network_measure(device, name: str, days: int) -> dict:
    """One of the small benchmark configurations (plain_60k: 60,000
    catchments, plain physics, daily runoff, the 3600 s dt cap; full_250k:
    250,000 catchments with full physics) routed through the public API over
    `days` daily intervals after one warm-up day, three ways on the same GPU:
    the interval graph, the persistent interval kernel, and the reference's
    own CUDA kernels (oracle/_ref, driven as CaMaFlood.step_advance drives
    them).  A sub-step here is a few microseconds of work, so launch and
    barrier costs decide.  The three end states are compared field by field.
    The reference has no dt cap, so on plain_60k its arm runs the capped count
    max(n, T / 3600 s) as a fixed count, as the parity test does."""
    import torch
    from cmfb200 import CaMaFlood, synthetic as syn
    from oracle import oracle as O, ref_cuda as RC
    cfg = syn.CONFIGS[name]
    net = syn.generate(cfg["spec"])
    cap_s = cfg.get("max_sub_step_seconds", 0.0)
    T = cfg["interval"]
    stream = torch.cuda.current_stream(device)
    out = {"catchments": net.num_catchments, "days": days, "warmup_days": 1,
           "modules": list(net.opened_modules)}
    states = {}
    for mode in ("graph", "persistent"):
        m = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
                      step_duration=T, max_sub_step_seconds=cap_s, persistent=(mode == "persistent"))
        run = [torch.as_tensor(syn.daily_runoff(net, d)[m.order]).to(device) for d in range(days + 1)]
        m.set_inputs(run[0])
        m.step_advance()
        cnt = torch.zeros(days, dtype=torch.int32, device=device)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for d in range(days):
            m.set_inputs(run[d + 1])
            m.step_advance()
            cnt[d].copy_(m.sub_step_counts()[0])
        e1.record(stream)
        torch.cuda.synchronize(device)
        m.check_status()
        subs = int(cnt.sum().item())
        ms = e0.elapsed_time(e1)
        out[mode] = {"value": net.num_catchments * subs / (ms / 1e3), "sub_steps": subs,
                     "us_per_substep": 1e3 * ms / subs}
        states[mode] = {k: v.cpu().numpy().copy() for k, v in m.state_tensors().items()}
        order = m.order
        m.close()
    out["persistent_over_graph"] = out["persistent"]["value"] / out["graph"]["value"]
    out["persistent_state_equal"] = all(np.array_equal(states["graph"][k], states["persistent"][k])
                                        for k in states["graph"])
    if RC.available():
        ref = RC.RefCuda(O.reference_fields(net.fields, net.opened_modules), net.opened_modules,
                         device=device)
        cap_n = int(round(T / cap_s)) if cap_s > 0 else 0
        run = [torch.as_tensor(syn.daily_runoff(net, d)).to(device) for d in range(days + 1)]

        def ref_step(d):
            ref.t["runoff"].copy_(run[d])
            if cap_n:
                n = max(ref.adaptive_sub_steps(T), cap_n)
                return ref.step_advance(T, adaptive=False, fixed_n=n)
            return ref.step_advance(T)

        ref_step(0)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        subs = 0
        for d in range(days):
            subs += ref_step(d + 1)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        out["reference_cuda"] = {"value": net.num_catchments * subs / (ms / 1e3), "sub_steps": subs,
                                 "us_per_substep": 1e3 * ms / subs}
        equal = True
        for k, a in states["graph"].items():
            b = ref.t[k].detach().cpu().numpy()
            if a.ndim == 1 and not k.startswith("bifurcation_"):
                b = b[order]
            equal = equal and bool(np.array_equal(a, b))
        out["reference_cuda"]["state_equal"] = equal
        best = max(out["graph"]["value"], out["persistent"]["value"])
        out["ours_best_over_reference_cuda"] = best / out["reference_cuda"]["value"]
        del ref
    return out


def adjoint_compare(device, days: int, checkpoint_every: int = 96, repeats: int = 5) -> dict:
    """Forward+adjoint against forward on the calibration window: the
    250k-catchment full-physics network (8,000 bifurcation paths, levees on
    20 % of cells, 500 reservoirs), fp64, daily forcing over `days`
    intervals, discharge at 500 cells with upstream area > 1000 km^2,
    relative-misfit loss against a run with river Manning x lognormal(0.2).
    Both are timed with CUDA events on the same GPU from the same spun-up
    state: three discarded warm-up pairs, then `repeats` interleaved repetitions,
    medians; the gradient run includes its checkpointed forward."""
    import torch
    from cmfb200 import CaMaFlood, synthetic as syn, topology
    from cmfb200.adjoint import AdjointRouting
    net = syn.generate(syn.CONFIGS["full_250k"]["spec"])
    model = CaMaFlood(device=device, input_proxy=net.fields,
                      opened_modules=net.opened_modules, precision="float64")
    model.set_inputs(torch.as_tensor(syn.daily_runoff(net, 0)[model.order]).to(device))
    model.step_advance()
    fx = model.export_fields()
    area = topology.accumulate_upstream(fx["downstream_idx"], fx["catchment_area"].astype(np.float64))
    rng = np.random.default_rng(4)
    cand = np.flatnonzero(area > 1.0e9)
    gauges = np.sort(rng.choice(cand, size=min(500, cand.size), replace=False))
    eng = AdjointRouting(model, gauges, checkpoint_every=checkpoint_every)
    forcing = torch.as_tensor(np.stack([syn.daily_runoff(net, 1 + d)[model.order]
                                        for d in range(days)]), dtype=torch.float64, device=device)
    params = eng.parameters()
    state0 = eng.initial_state()
    truth = dict(params)
    truth["river_manning"] = params["river_manning"] * torch.as_tensor(
        np.exp(0.2 * rng.standard_normal(eng.N)), device=device)
    q_obs, _ = eng.forward_only(truth, forcing, state0)
    stream = torch.cuda.current_stream(device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def fwd():
        return eng.forward_only(params, forcing, state0)

    def fwd_adj():
        p = {k: v.clone().requires_grad_(True) for k, v in params.items()}
        f = forcing.clone().requires_grad_(True)
        q, _ = eng.window(p, f, state0)
        loss = (((q - q_obs) / q_obs) ** 2).sum()
        return torch.autograd.grad(loss, [p["river_manning"], p["river_height"],
                                          p["river_width"], f])

    for _ in range(3):                        # warm-up (allocations, lazy init, clocks)
        fwd()
        fwd_adj()
    torch.cuda.synchronize(device)
    # interleaved repetitions, medians reported (single runs vary by a few
    # per cent with the GPU's power state)
    reps = max(1, int(repeats))
    tf, ta = [], []
    for _ in range(reps):
        ev[0].record(stream)
        fwd()
        ev[1].record(stream)
        torch.cuda.synchronize(device)
        ev[2].record(stream)
        fwd_adj()
        ev[3].record(stream)
        torch.cuda.synchronize(device)
        tf.append(ev[0].elapsed_time(ev[1]) / 1e3)
        ta.append(ev[2].elapsed_time(ev[3]) / 1e3)
    t_fwd = statistics.median(tf)
    t_adj = statistics.median(ta)
    # the product's own fp64 forward (interval graphs) over the same window
    snap = {k: v.clone() for k, v in model.state_tensors().items()}
    b = model.base
    for k in ("river_manning", "flood_manning", "river_height", "river_width"):
        getattr(b, k).copy_(params[k])

    def product_fwd():
        for k, v in model.state_tensors().items():
            v.copy_(snap[k])
        for d in range(days):
            model.set_inputs(forcing[d])
            model.step_advance()

    product_fwd()
    torch.cuda.synchronize(device)
    tp = []
    for _ in range(reps):
        ev[0].record(stream)
        product_fwd()
        ev[1].record(stream)
        torch.cuda.synchronize(device)
        tp.append(ev[0].elapsed_time(ev[1]) / 1e3)
    t_prod = statistics.median(tp)
    # the product's mixed-precision forward (fp32 fluxes, fp64 storage: the
    # reference's default) over the same window from the same state
    mixed = CaMaFlood(device=device, input_proxy=net.fields,
                      opened_modules=net.opened_modules, precision="float32")
    for k, v in mixed.state_tensors().items():
        v.copy_(snap[k].to(v.dtype))
    mb = mixed.base
    for k in ("river_manning", "flood_manning", "river_height", "river_width"):
        getattr(mb, k).copy_(params[k].to(getattr(mb, k).dtype))
    snap_m = {k: v.clone() for k, v in mixed.state_tensors().items()}
    forcing32 = forcing.float()

    def mixed_fwd():
        for k, v in mixed.state_tensors().items():
            v.copy_(snap_m[k])
        for d in range(days):
            mixed.set_inputs(forcing32[d])
            mixed.step_advance()

    mixed_fwd()
    torch.cuda.synchronize(device)
    tm = []
    for _ in range(reps):
        ev[0].record(stream)
        mixed_fwd()
        ev[1].record(stream)
        torch.cuda.synchronize(device)
        tm.append(ev[0].elapsed_time(ev[1]) / 1e3)
    t_mixed = statistics.median(tm)
    mixed.close()
    # sub-step count of the window (the CFL counts of the primal run)
    _, _, counts, _, _ = eng._forward(params["river_manning"], params["flood_manning"],
                                      params["river_height"], params["river_width"], forcing,
                                      state0, keep_checkpoints=False)
    subs = int(sum(counts))
    n_lev = model.levee.num_levees if model.levee is not None else 0
    n_res = model.reservoir.num_reservoirs if model.reservoir is not None else 0
    model.close()
    n = eng.N
    peak, peak_kind = measured_peak()
    b_fwd = fp64_algorithmic_bytes(n, eng.P, n_lev, n_res)
    b_adj = adjoint_algorithmic_bytes(n, eng.P, n_lev, n_res, eng.state_len, eng.slot_len,
                                      eng.n_grad)
    ach_fwd = b_fwd * subs / t_fwd / 1e9
    ach_adj = b_adj * subs / t_adj / 1e9
    each = [a / f for a, f in zip(ta, tf)]
    return {"fwd_value": n * subs / t_fwd, "fwd_adj_value": n * subs / t_adj, "unit": UNIT,
            "roofline": {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_kind": peak_kind,
                         "fwd_bytes_per_substep": b_fwd, "fwd_adj_bytes_per_substep": b_adj,
                         "fwd_achieved": ach_fwd, "fwd_frac": ach_fwd / peak,
                         "fwd_adj_achieved": ach_adj, "fwd_adj_frac": ach_adj / peak},
            "fwd_adj_over_fwd": t_adj / t_fwd,
            "repeats": reps, "fwd_adj_over_fwd_each": each,
            "fwd_adj_over_fwd_spread": (max(each) - min(each)) / statistics.median(each),
            "fwd_s_each": tf, "fwd_adj_s_each": ta,
            "product_fwd_value": n * subs / t_prod, "fwd_adj_over_product_fwd": t_adj / t_prod,
            "fwd_adj_over_mixed_product_fwd": t_adj / t_mixed,
            "mixed_product_fwd_ms": t_mixed * 1e3,
            "catchments": n, "sub_steps": subs,
            "days": days, "checkpoint_every": checkpoint_every, "gauges": int(gauges.size),
            "dtype": "f64",
            "workload": "full-physics 250k network, fp64, daily forcing, gradients w.r.t. "
                        "river Manning, river height, river width and runoff; fwd = the same "
                        "primal kernels without checkpoints; product_fwd = CaMaFlood.step_advance "
                        "in fp64 (interval graphs) over the same window; mixed_product_fwd = the "
                        "same in the reference's mixed precision (fp32 fluxes, fp64 storage)"}


def adjoint_fd_check(device, days: int, cells: int, seed: int = 5) -> dict:
    """Central finite differences of the calibration loss on the 250k
    full-physics network at `cells` random cells per parameter (river and
    floodplain Manning, river height, river width, runoff of the first day)
    against the CUDA adjoint: h = 1e-4 relative, retried at 1e-6 where the
    step crosses a branch of the piecewise physics; a cell passes when
    |ad - fd| <= 1e-3 * max(|ad|, 1e-3 * max|grad of that field|)."""
    import torch
    from cmfb200 import CaMaFlood, synthetic as syn
    from cmfb200.adjoint import AdjointRouting, PARAMS
    net = syn.generate(syn.CONFIGS["full_250k"]["spec"])
    model = CaMaFlood(device=device, input_proxy=net.fields,
                      opened_modules=net.opened_modules, precision="float64")
    model.set_inputs(torch.as_tensor(syn.daily_runoff(net, 0)[model.order]).to(device))
    model.step_advance()
    rng = np.random.default_rng(seed)
    gauges = np.sort(rng.choice(model.num_catchments, size=500, replace=False))
    eng = AdjointRouting(model, gauges)
    forcing = torch.as_tensor(np.stack([syn.daily_runoff(net, 1 + d)[model.order]
                                        for d in range(days)]), dtype=torch.float64, device=device)
    params = eng.parameters()
    state0 = eng.initial_state()
    truth = dict(params)
    truth["river_manning"] = params["river_manning"] * torch.as_tensor(
        np.exp(0.2 * rng.standard_normal(eng.N)), device=device)
    q_obs, _ = eng.forward_only(truth, forcing, state0)

    def loss(q):
        return (((q - q_obs) / q_obs) ** 2).sum()

    p = {k: v.clone().requires_grad_(True) for k, v in params.items()}
    f = forcing.clone().requires_grad_(True)
    q, _ = eng.window(p, f, state0)
    grads = torch.autograd.grad(loss(q), [p[k] for k in PARAMS] + [f])

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
            vals.append(float(loss(eng.forward_only(pp, ff, state0)[0])))
        return (vals[0] - vals[1]) / (2 * h)

    passed, total, worst, at_small_h = 0, 0, 0.0, 0
    for name, g in zip(list(PARAMS) + ["runoff"], grads):
        flat = (g[0] if name == "runoff" else g).detach()
        gmax = float(flat.abs().max())
        for c in rng.choice(eng.N, size=cells, replace=False).tolist():
            ad = flat[c].item()
            scale = max(abs(ad), 1e-3 * gmax)
            e1 = abs(ad - fd(name, c, 1e-4)) / scale
            err = e1 if e1 <= 1e-3 else min(e1, abs(ad - fd(name, c, 1e-6)) / scale)
            at_small_h += int(e1 > 1e-3 and err <= 1e-3)
            passed += int(err <= 1e-3)
            total += 1
            worst = max(worst, err)
    model.close()
    return {"cells_per_field": cells, "fields": list(PARAMS) + ["runoff"], "passed": passed,
            "total": total, "passed_without_retry": passed - at_small_h,
            "passed_at_h_1e-6": at_small_h, "max_scaled_error": worst,
            "days": days, "catchments": eng.N}


REF_PHASES = ("outflow", "reservoir", "bif_outflow", "inflow", "bif_inflow", "flood_stage",
              "levee_stage")


def reference_cuda_measure(device, net, cfg, args, dev_forcing_in, our_state, order) -> dict:
    """The reference's own CUDA kernels on the same workload and GPU: the
    cmfgpu/phys/cuda/*.cu sources compiled unmodified for sm_100a
    (oracle/_ref), driven as CaMaFlood.step_advance drives them
    (cmfgpu/models/cama_flood_model.py:104-173): per interval the CFL kernel
    and one .item() host sync, then per sub-step up to seven launches
    (outflow, reservoir, bifurcation outflow, inflow, bifurcation inflow,
    flood stage, levee stage) with fp64 atomic scatters.  It routes the same
    spin-up and warm-up intervals and then the timed intervals from the same
    initial state; its state after them is compared with ours field by
    field."""
    import torch
    from oracle import oracle as O, ref_cuda as RC
    if not RC.available():
        return {"unavailable": "oracle/_ref (the reference CUDA kernels) is not built"}
    fields = O.reference_fields(net.fields, net.opened_modules)
    ref = RC.RefCuda(fields, net.opened_modules, device=device)
    interval = cfg["interval"]
    runoff = ref.t["runoff"]

    def set_runoff(x):
        runoff.copy_(x)

    spin_up(net, cfg, args.spinup_days, device, None, set_runoff,
            lambda: ref.step_advance(interval))
    steps = dev_forcing_in.shape[0] - args.warmup
    for k in range(args.warmup):
        set_runoff(dev_forcing_in[k])
        ref.step_advance(interval)
    stream = torch.cuda.current_stream(device)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    subs = 0
    e0.record(stream)
    for k in range(args.warmup, args.warmup + steps):
        set_runoff(dev_forcing_in[k])
        subs += ref.step_advance(interval)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    # state after the same intervals: ours (model order) against the reference
    mism = {}
    for k, v in our_state.items():
        r = ref.t[k]
        a = v.cpu().numpy()
        b = r.detach().cpu().numpy()
        if a.ndim == 1:                       # catchment fields: input -> model order
            b = b[order]
        mism[k] = int(np.count_nonzero(a != b))
    # per-kernel device times of one more interval (events around each launch)
    mods = set(net.opened_modules)
    set_runoff(dev_forcing_in[-1])
    n = ref.adaptive_sub_steps(interval)
    ref.t["time_step"].fill_(interval / n)
    calls = [("outflow", ref.outflow, True), ("reservoir", ref.reservoir, "reservoir" in mods),
             ("bif_outflow", ref.bif_outflow, "bifurcation" in mods),
             ("inflow", ref.inflow, True), ("bif_inflow", ref.bif_inflow, "bifurcation" in mods),
             ("flood_stage", ref.flood_stage, True), ("levee_stage", ref.levee_stage, "levee" in mods)]
    calls = [(nm, fn) for nm, fn, on in calls if on]
    evs = []
    for _ in range(n):
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(calls) + 1)]
        marks[0].record(stream)
        for j, (_, fn) in enumerate(calls):
            fn()
            marks[j + 1].record(stream)
        evs.append(marks)
    torch.cuda.synchronize(device)
    per = {nm: float(np.mean([m[j].elapsed_time(m[j + 1]) for m in evs]))
           for j, (nm, _) in enumerate(calls)}
    value = net.num_catchments * subs / (ms / 1e3)
    del ref
    torch.cuda.empty_cache()
    return {"value": value, "unit": UNIT, "ms_per_step": ms / steps, "sub_steps_timed": subs,
            "ms_per_substep_kernels": per, "ms_per_substep_kernel_sum": sum(per.values()),
            "launches_per_substep": len(calls),
            "state_mismatches_vs_ours": mism,
            "state_equal": all(v == 0 for v in mism.values()),
            "what": "the reference's cmfgpu/phys/cuda kernels, unmodified, compiled for sm_100a "
                    "(oracle/_ref), driven per interval as CaMaFlood.step_advance does (CFL kernel "
                    "+ .item(), then up to 7 launches per sub-step, fp64 atomics), same intervals, "
                    "same initial state, same GPU; device time by CUDA events"}


def run_reference(args) -> None:
    """The reference algorithm's CPU restatement on all host cores (rank 0
    only).  The reference ships no CPU path, so this is the oracle port
    (oracle/cmf_oracle.c, OpenMP).  The network is built with the oracle's
    topology helpers and the product library is never loaded; the line lists
    the in-tree libraries this process mapped."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O, topology as OT
    net, cfg = build_workload(args.workload, 0, topo=OT)
    fields = O.reference_fields(net.fields, net.opened_modules)
    orc = O.Oracle(fields, net.opened_modules)
    threads = O.max_threads()
    runoff = runoff_series(net, cfg, 1)[0]
    orc.set_runoff(runoff)
    n = orc.adaptive_sub_steps(cfg["interval"], cfg.get("max_sub_step_seconds", 0.0))
    orc.set_time_step(cfg["interval"] / max(n, 1), cfg["interval"])
    # one step = a bounded sample of sub-steps of the interval
    t0 = time.perf_counter()
    orc.substep()
    one = time.perf_counter() - t0
    per_step = max(1, int(4.0 / max(one, 1e-6)))
    per_step = min(per_step, n)
    for _ in range(args.warmup):
        for _ in range(per_step):
            orc.substep()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for _ in range(per_step):
            orc.substep()
    el = time.perf_counter() - t0
    value = net.num_catchments * per_step * args.steps / el
    sample = (f"{per_step} of the interval's {n} sub-steps per step from the cold start, "
              f"{net.num_catchments}-catchment {args.workload} network, {threads} OpenMP threads")
    libs = loaded_native_libraries()
    if any("libcmfb200" in x for x in libs):
        raise RuntimeError(f"the reference arm loaded the product library: {libs}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 flux / f64 storage",
        "data": "synthetic (seeded generator, no CaMa maps)",
        "config": workload_config(args, net, cfg, max(1, int(os.environ.get("WORLD_SIZE", "1")))),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_libraries": libs,
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist
    from cmfb200 import CaMaFlood, _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    net, cfg = build_workload(args.workload, rank)
    full = len(net.opened_modules) > 2
    model = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
                      step_duration=cfg["interval"],
                      max_sub_step_seconds=cfg.get("max_sub_step_seconds", 0.0),
                      BLOCK_SIZE=args.block or 256)
    N = net.num_catchments
    P = model.bifurcation.num_bifurcation_paths if model.bifurcation is not None else 0
    Lv = model.levee.num_levees if model.levee is not None else 0
    R = model.reservoir.num_reservoirs if model.reservoir is not None else 0
    total = args.warmup + args.steps
    order = model.order
    order_dev = torch.as_tensor(order, device=device)

    def sync_all():
        torch.cuda.synchronize(device)
        if world > 1:
            dist.barrier()

    # ---- spin-up: route the first simulated days (untimed, graphs) ------------
    spun = spin_up(net, cfg, args.spinup_days, device, order, model.set_inputs,
                   model.step_advance)
    forcing_in = runoff_series(net, cfg, total, start=spun)           # input order
    host = torch.from_numpy(np.ascontiguousarray(forcing_in[:, order])).pin_memory()
    dev_forcing = host.to(device)                                      # model order
    counts = torch.zeros(total, dtype=torch.int32, device=device)

    tuned = None
    if args.block == 0:
        # block size chosen by the autotuner on this network (outside the timed
        # region; the state is restored afterwards)
        model.set_inputs(dev_forcing[0])
        tuned = model.autotune_block_size()

    # warm-up (also builds the interval graph)
    for k in range(args.warmup):
        model.set_inputs(dev_forcing[k])
        model.step_advance()
    sync_all()

    # ---- timed region: forcing resident in HBM --------------------------------
    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            gpu_index = int(vis.split(",")[local])
        except ValueError:
            pass
    sampler = ClockSampler(gpu_index)
    time.sleep(0.3)
    stream = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sync_all()
    e0.record(stream)
    for k in range(args.warmup, total):
        model.set_inputs(dev_forcing[k])
        model.step_advance()
        counts[k].copy_(model.sub_step_counts()[0])
    e1.record(stream)
    sync_all()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    substeps = int(counts[args.warmup:].sum().item())
    per_sub = 4 if Lv > 0 else 3                 # momentum, limit, stage (+ levee)
    launches = 4 * args.steps + per_sub * substeps   # + begin, cfl, plan, end per interval
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    w = torch.tensor([N * substeps], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    value = float(w.item()) / (ms_max / 1e3)
    # the state the timed intervals left, for the reference-CUDA comparison
    our_state = {k: v.clone() for k, v in model.state_tensors().items()}
    flooded = float((model.base.flood_storage > 0).double().mean().item())
    prot = (float((model.base.protected_storage > 0).double().mean().item())
            if model.levee is not None else 0.0)

    # ---- per-kernel timing (one interval through direct launches) -------------
    kern = {"momentum": [], "limit": [], "stage": [], "levee": []}
    model.set_inputs(dev_forcing[total - 1])
    model.compute_adaptive_time_step()
    n_int = int(model.sub_step_counts()[0].item())
    evs = []
    for k in range(n_int):
        a, b, c, d, e = (torch.cuda.Event(enable_timing=True) for _ in range(5))
        a.record(stream)
        model.launch_substep_kernel(k, _lib.PART_MOMENTUM)
        b.record(stream)
        model.launch_substep_kernel(k, _lib.PART_LIMIT)
        c.record(stream)
        model.launch_substep_kernel(k, _lib.PART_STAGE)
        d.record(stream)
        model.launch_substep_kernel(k, _lib.PART_LEVEE)
        e.record(stream)
        evs.append((a, b, c, d, e))
    model.launch_substep_kernel(n_int, _lib.PART_END)
    torch.cuda.synchronize(device)
    for a, b, c, d, e in evs:
        kern["momentum"].append(a.elapsed_time(b))
        kern["limit"].append(b.elapsed_time(c))
        kern["stage"].append(c.elapsed_time(d))
        kern["levee"].append(d.elapsed_time(e))
    t_mom = float(np.mean(kern["momentum"]))
    t_lim = float(np.mean(kern["limit"]))
    t_stage = float(np.mean(kern["stage"]))
    t_lev = float(np.mean(kern["levee"]))
    t_sub = t_mom + t_lim + t_stage + t_lev
    alg = algorithmic_bytes(N, P, Lv, R, full)
    peak, peak_kind = measured_peak()
    achieved = alg / (t_sub / 1e3) / 1e9
    traffic = None
    traffic_src = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            tj = json.loads(tfile.read_text())
            if tj.get("workload") == args.workload:
                traffic = tj.get("bytes_per_substep")
                traffic_src = tj.get("source")
        except Exception:
            traffic = None

    # ---- e2e through the public API with host buffers --------------------------
    # Every interval's runoff crosses from pinned host memory (InputPrefetcher:
    # the copy of interval k+1 overlaps the routing of k) and every interval's
    # gauge discharge comes back to the host, read by the caller while the
    # next interval routes.
    from cmfb200.prefetch import InputPrefetcher
    gauges = torch.as_tensor(np.linspace(0, N - 1, 1000).astype(np.int64), device=device)
    out_host = torch.empty((args.steps, gauges.numel()), dtype=torch.float32).pin_memory()
    prefetch = InputPrefetcher(model)
    done = [torch.cuda.Event() for _ in range(args.steps)]
    gauge_sum = 0.0
    sync_all()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    e2e_sub = torch.zeros(args.steps, dtype=torch.int32, device=device)
    prefetch.submit(host[args.warmup])
    for j, k in enumerate(range(args.warmup, total)):
        if k + 1 < total:
            prefetch.submit(host[k + 1])                   # pinned H2D, overlapped
        prefetch.set_inputs()
        model.step_advance()
        e2e_sub[j].copy_(model.sub_step_counts()[0])
        out_host[j].copy_(model.base.river_outflow.index_select(0, gauges), non_blocking=True)
        done[j].record(stream)
        if j >= 1:
            done[j - 1].synchronize()                      # the caller reads interval j-1
            gauge_sum += float(out_host[j - 1].sum())
    done[args.steps - 1].synchronize()
    gauge_sum += float(out_host[args.steps - 1].sum())
    h1.record(stream)
    sync_all()
    e2e_ms = h0.elapsed_time(h1)
    e2e_work = N * int(e2e_sub.sum().item())
    t2 = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
    w2 = torch.tensor([e2e_work], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        dist.all_reduce(w2, op=dist.ReduceOp.SUM)
    e2e_value = float(w2.item()) / (float(t2.item()) / 1e3)
    model.check_status()

    stats = None
    if args.statistics:
        # same forcing as the timed region (state has moved on; sub-step counts may differ)
        stats = statistics_overhead(model, dev_forcing, args.warmup, args.steps, ms, substeps)

    forcing_leg = None
    if world == 1 and args.forcing_steps > 0:
        forcing_leg = forcing_measure(device, net, model.base.catchment_id.cpu().numpy(),
                                      steps=args.forcing_steps)

    ref_cuda = None
    if world == 1 and args.reference_cuda:
        model.close()
        del dev_forcing
        dev_in = torch.as_tensor(forcing_in).to(device)
        ref_cuda = reference_cuda_measure(device, net, cfg, args, dev_in, our_state, order)
        del dev_in
        if "value" in ref_cuda:
            ref_cuda["ours_over_reference_cuda"] = value / ref_cuda["value"]
            ref_cuda["kernel_sum_ratio"] = ref_cuda["ms_per_substep_kernel_sum"] / t_sub
    del our_state

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(net, cfg, None)

    ensemble = None
    if world == 1 and args.ensemble_members > 0:
        model.close()
        ensemble = ensemble_compare(device, args.ensemble_members, args.ensemble_catchments,
                                    member_tile=args.ensemble_member_tile,
                                    block=args.ensemble_block, days=args.ensemble_days)

    small = None
    if world == 1 and args.small_networks:
        model.close()
        small = {"plain_60k": small_network_measure(device, "plain_60k", 29),
                 "full_250k": small_network_measure(device, "full_250k", 10)}

    adjoint = None
    if world == 1 and args.adjoint_days > 0:
        model.close()
        adjoint = adjoint_compare(device, args.adjoint_days, repeats=args.adjoint_repeats)
        if args.adjoint_fd_cells > 0:
            adjoint["fd_check"] = adjoint_fd_check(device, args.adjoint_fd_days, args.adjoint_fd_cells)

    if world > 1:
        dist.barrier()
    if rank == 0:
        config = workload_config(args, net, cfg, world)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 storage", "data": "synthetic (seeded generator, no CaMa maps)",
            "config": config,
            "run": {"sub_steps_timed": substeps, "block": model.block_size,
                    "block_tuned": tuned is not None, "spinup_intervals": spun,
                    "flooded_cell_fraction": flooded, "protected_cell_fraction": prot},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": N * 4,
                    "d2h_bytes_per_step": int(gauges.numel()) * 4,
                    "path": "InputPrefetcher.submit (pinned H2D on a copy stream) -> set_inputs -> "
                            "step_advance -> gauge D2H read by the host each interval",
                    "gauge_discharge_sum": gauge_sum},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                         "peak_kind": peak_kind, "kernel": "sub-step (k_momentum + k_limit + k_stage + k_levee)",
                         "algorithmic_bytes_per_substep": alg,
                         "ms_momentum": t_mom, "ms_limit": t_lim, "ms_stage": t_stage,
                         "ms_levee": t_lev},
            "reference_cuda": ref_cuda,
            "cpu_baseline": cpu,
            "ensemble": ensemble,
            "small_networks": small,
            "adjoint": adjoint,
            "forcing": forcing_leg,
            "statistics": stats,
            "clocks": clocks,
            "gpu_launches": launches,
            "native_libraries": loaded_native_libraries(),
        }
        print(json.dumps(line), flush=True)
    model.close()
    if world > 1:
        dist.destroy_process_group()


def probe_ensemble(args) -> None:
    """The member-batched form of probe_kernels: the ensemble workload
    (`--ensemble-members` members of `--ensemble-catchments` catchments in 500
    basins, runoff and river Manning perturbed per member, member tile
    `--ensemble-member-tile`, `--ensemble-block`-thread CTAs) routed for
    `--spinup-days` daily intervals, then each sub-step kernel launched once
    inside the NVTX range "probe"."""
    import torch
    from cmfb200 import CaMaFlood, synthetic as syn, _lib
    device = torch.device("cuda", 0)
    members = args.ensemble_members
    net = syn.generate_basins(500, args.ensemble_catchments, seed=3)
    rfac, mfac = syn.ensemble_factors(net.num_catchments, members, seed=3)
    manning = (net.fields["river_manning"][:, None] * mfac).astype(np.float32)
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=["base", "adaptive_time"],
                    num_members=members, batched_fields={"river_manning": manning},
                    BLOCK_SIZE=args.ensemble_block)
    ens.set_member_tile(max(1, args.ensemble_member_tile))
    order = ens.order
    rf = torch.as_tensor(rfac[order]).to(device)

    def runoff(d):
        return (torch.as_tensor(syn.daily_runoff(net, d)[order]).to(device)[:, None] * rf).contiguous()

    for d in range(args.spinup_days):
        ens.set_inputs(runoff(d))
        ens.step_advance()
    ens.set_inputs(runoff(args.spinup_days))
    ens.compute_adaptive_time_step()
    torch.cuda.synchronize(device)
    parts = [("k_momentum", _lib.PART_MOMENTUM), ("k_limit", _lib.PART_LIMIT),
             ("k_stage", _lib.PART_STAGE)]
    torch.cuda.nvtx.range_push("probe")
    for _, part in parts:
        ens.launch_substep_kernel(0, part)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(device)
    ens.check_status()
    print(json.dumps({"probe": [p for p, _ in parts], "members": members,
                      "catchments": net.num_catchments, "spinup_days": args.spinup_days,
                      "member_tile": ens.member_tile, "block": ens.block_size,
                      "flooded_fraction": float((ens.base.flood_storage > 0).double().mean().item())}),
          flush=True)
    ens.close()


def probe_kernels(args) -> None:
    """One launch of each sub-step kernel on the spun-up workload, outside the
    interval graph and inside an NVTX range named "probe", for a profiler to
    capture (ncu --nvtx --nvtx-include "probe/").  Prints what it launched."""
    import torch
    from cmfb200 import CaMaFlood, _lib
    device = torch.device("cuda", 0)
    net, cfg = build_workload(args.workload, 0)
    model = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
                      step_duration=cfg["interval"],
                      max_sub_step_seconds=cfg.get("max_sub_step_seconds", 0.0),
                      BLOCK_SIZE=args.block or 64)
    spun = spin_up(net, cfg, args.spinup_days, device, model.order, model.set_inputs,
                   model.step_advance)
    model.set_inputs(torch.as_tensor(runoff_series(net, cfg, 1, start=spun)[0][model.order]).to(device))
    model.compute_adaptive_time_step()
    torch.cuda.synchronize(device)
    parts = [("k_momentum", _lib.PART_MOMENTUM), ("k_limit", _lib.PART_LIMIT),
             ("k_stage", _lib.PART_STAGE)]
    if model.levee is not None:
        parts.append(("k_levee", _lib.PART_LEVEE))
    torch.cuda.nvtx.range_push("probe")
    for _, part in parts:
        model.launch_substep_kernel(0, part)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(device)
    model.check_status()
    print(json.dumps({"probe": [p for p, _ in parts], "workload": args.workload,
                      "catchments": net.num_catchments, "spinup_intervals": spun,
                      "block": model.block_size,
                      "flooded_cell_fraction": float((model.base.flood_storage > 0).double().mean().item())}),
          flush=True)
    model.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="full_6m")
    ap.add_argument("--block", type=int, default=0,
                    help="threads per CTA; 0 lets the autotuner choose")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble-members", type=int, default=64,
                    help="members of the batched-vs-looped comparison (0 skips it)")
    ap.add_argument("--adjoint-days", type=int, default=30,
                    help="daily intervals of the forward+adjoint comparison (0 = skip)")
    ap.add_argument("--adjoint-repeats", type=int, default=5,
                    help="interleaved timed repetitions of the adjoint comparison")
    ap.add_argument("--adjoint-fd-cells", type=int, default=50,
                    help="random cells per parameter of a finite-difference check of the "
                         "adjoint on the 250k network (0 = skip)")
    ap.add_argument("--adjoint-fd-days", type=int, default=3,
                    help="window length of that check")
    ap.add_argument("--forcing-steps", type=int, default=24,
                    help="steps per chunk of the gridded-runoff forcing map leg (0 = skip)")
    ap.add_argument("--no-statistics", dest="statistics", action="store_false",
                    help="skip the output-statistics overhead leg")
    ap.add_argument("--ensemble-catchments", type=int, default=6_000_000,
                    help="catchments per member of that comparison (the benchmark's ensemble "
                         "workload: ~6M in 500 basins)")
    ap.add_argument("--ensemble-member-tile", type=int, default=16,
                    help="members of a catchment per thread in the batched model "
                         "(0: autotuned block size and tile); 16 with 64-thread CTAs is "
                         "the fastest pair measured at 64 members x 6M catchments")
    ap.add_argument("--ensemble-days", type=int, default=5,
                    help="simulated days of the ensemble comparison")
    ap.add_argument("--spinup-days", type=int, default=9,
                    help="simulated days routed before the timed intervals (a warm, flooded state)")
    ap.add_argument("--no-reference-cuda", dest="reference_cuda", action="store_false",
                    help="skip timing the reference's own CUDA kernels on the same workload")
    ap.add_argument("--no-small-networks", dest="small_networks", action="store_false",
                    help="skip the small-configuration leg (60k plain and 250k full physics: "
                         "interval graph, persistent kernel and the reference's CUDA kernels)")
    ap.add_argument("--probe-ensemble", action="store_true",
                    help="with --probe-kernels: probe the member-batched kernels of the ensemble "
                         "workload instead")
    ap.add_argument("--probe-kernels", action="store_true",
                    help="launch each sub-step kernel once on the spun-up workload inside an "
                         "NVTX range 'probe' (for a profiler) and exit")
    ap.add_argument("--ensemble-block", type=int, default=64,
                    help="threads per CTA of the batched model")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.probe_kernels and args.probe_ensemble:
        probe_ensemble(args)
    elif args.probe_kernels:
        probe_kernels(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
