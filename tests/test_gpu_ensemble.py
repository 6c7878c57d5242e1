"""Member-innermost ensemble: one launch per phase for M members, each with
its own CFL sub-step count and dt.  Every member of the batched run must equal
(bit for bit) a plain single-member run on that member's inputs."""
import numpy as np
import pytest
import torch

from cmfb200 import CaMaFlood, synthetic as syn

pytestmark = pytest.mark.gpu


def _plain(net, manning, device, precision="float32"):
    f = dict(net.fields)
    f["river_manning"] = manning
    return CaMaFlood(device=device, input_proxy=f, opened_modules=["base", "adaptive_time"],
                     precision=precision)


# member counts that are and are not powers of two, with and without a member
# tile, in fp32 and fp64
@pytest.mark.parametrize("members,precision", [(4, "float32"), (3, "float32"), (8, "float32"),
                                               (16, "float32"), (8, "float64")])
def test_batched_members_equal_plain_runs(members, precision, device):
    net = syn.generate_basins(40, 30_000, seed=9)
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=9)
    real = np.float32 if precision == "float32" else np.float64
    manning = (net.fields["river_manning"][:, None] * mfac).astype(real)
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=["base", "adaptive_time"],
                    num_members=members, batched_fields={"river_manning": manning},
                    precision=precision)
    if members % 4 == 0 and members > 4:
        ens.set_member_tile(4)
    plains = [_plain(net, np.ascontiguousarray(manning[:, m]), device, precision)
              for m in range(members)]
    order = ens.order
    counts = []
    for day in range(2):
        r = syn.daily_runoff(net, day)
        rm = (r[:, None] * rfac).astype(real)
        ens.set_inputs(torch.as_tensor(rm[order]).to(device))
        ens.step_advance()
        counts.append(ens.sub_step_counts().cpu().numpy().copy())
        for m, p in enumerate(plains):
            assert np.array_equal(p.order, order)
            p.set_inputs(torch.as_tensor(np.ascontiguousarray(rm[:, m])[order]).to(device))
            p.step_advance()
            assert int(p.sub_step_counts()[0].item()) == int(counts[-1][m])
    torch.cuda.synchronize()
    # members genuinely differ (different Manning and runoff, different dt)
    assert len({tuple(c) for c in counts}) >= 1
    a = ens.state_tensors()
    for m, p in enumerate(plains):
        b = p.state_tensors()
        for k in b:
            np.testing.assert_array_equal(a[k][..., m].cpu().numpy(), b[k].cpu().numpy(),
                                          err_msg=f"member {m} field {k}")
    ens.check_status()


@pytest.mark.parametrize("batched", [("river_manning",), ("river_height", "river_width")])
def test_full_physics_members_equal_plain_runs(batched, device):
    """Levees, bifurcation paths and reservoirs with per-member parameters:
    member-batched river geometry makes the levee kernel read the cells'
    geometry per member instead of the plan's levee-indexed copies."""
    members = 4
    net = syn.generate(syn.NetworkSpec(20_000, seed=19, bifurcation_paths=150, levee_fraction=0.25,
                                       reservoirs=12))
    n = net.num_catchments
    rng = np.random.default_rng(19)
    per = {k: (net.fields[k][:, None] * rng.uniform(0.85, 1.15, size=(n, members))).astype(np.float32)
           for k in batched}
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
                    num_members=members, batched_fields=per)
    plains = []
    for m in range(members):
        f = dict(net.fields)
        for k, v in per.items():
            f[k] = np.ascontiguousarray(v[:, m])
        plains.append(CaMaFlood(device=device, input_proxy=f, opened_modules=net.opened_modules))
    order = ens.order
    for day in range(2):
        r = syn.daily_runoff(net, day)
        ens.set_inputs(torch.as_tensor(np.repeat(r[order, None], members, axis=1)).to(device))
        ens.step_advance()
        for p in plains:
            assert np.array_equal(p.order, order)
            p.set_inputs(torch.as_tensor(r[order]).to(device))
            p.step_advance()
    torch.cuda.synchronize()
    a = ens.state_tensors()
    for m, p in enumerate(plains):
        b = p.state_tensors()
        for k in b:
            np.testing.assert_array_equal(a[k][..., m].cpu().numpy(), b[k].cpu().numpy(),
                                          err_msg=f"member {m} field {k}")
    ens.check_status()


@pytest.mark.parametrize("width", [2, 4])
def test_member_tile_changes_no_result(width, device):
    """A thread per W consecutive members of a cell (cmf_plan_set_member_tile)
    routes exactly as a thread per member: levees, bifurcation paths and
    reservoirs, members with their own Manning and runoff, the tile switched
    between days."""
    members = 8
    net = syn.generate(syn.NetworkSpec(20_000, seed=29, bifurcation_paths=150, levee_fraction=0.25,
                                       reservoirs=12))
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=29)
    per = {"river_manning": (net.fields["river_manning"][:, None] * mfac).astype(np.float32)}
    kw = dict(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
              num_members=members, batched_fields=per)
    ref, tiled = CaMaFlood(**kw), CaMaFlood(**kw)
    tiled.set_member_tile(width)
    order = ref.order
    for day in range(3):
        r = syn.daily_runoff(net, day)
        rm = torch.as_tensor((r[:, None] * rfac).astype(np.float32)[order]).to(device)
        for m in (ref, tiled):
            m.set_inputs(rm)
            m.step_advance()
        if day == 1:
            tiled.set_member_tile(1)
            tiled.set_member_tile(width)
        torch.cuda.synchronize()
        a, b = ref.state_tensors(), tiled.state_tensors()
        for k in a:
            np.testing.assert_array_equal(b[k].cpu().numpy(), a[k].cpu().numpy(),
                                          err_msg=f"day {day} field {k}")
    assert tiled.member_tile == width
    tiled._rebuild_plan(128)                  # a rebuilt plan keeps the tile
    assert tiled.member_tile == width
    with pytest.raises(ValueError):
        tiled.set_member_tile(3)
    tiled.check_status()


@pytest.mark.parametrize("width", [1, 2])
def test_fp64_full_physics_members_equal_plain_runs(width, device):
    """The fp64 kernels (precision="float64") batched over members, with and
    without a member tile, against plain fp64 runs of each member."""
    members = 4
    net = syn.generate(syn.NetworkSpec(8_000, seed=37, bifurcation_paths=80, levee_fraction=0.25,
                                       reservoirs=8))
    n = net.num_catchments
    rfac, mfac = syn.ensemble_factors(n, members, seed=37)
    manning = (net.fields["river_manning"][:, None] * mfac).astype(np.float64)
    ens = CaMaFlood(device=device, input_proxy=net.fields, opened_modules=net.opened_modules,
                    num_members=members, batched_fields={"river_manning": manning},
                    precision="float64")
    ens.set_member_tile(width)
    plains = []
    for m in range(members):
        f = dict(net.fields)
        f["river_manning"] = np.ascontiguousarray(manning[:, m])
        plains.append(CaMaFlood(device=device, input_proxy=f, opened_modules=net.opened_modules,
                                precision="float64"))
    order = ens.order
    for day in range(2):
        rm = (syn.daily_runoff(net, day)[:, None] * rfac)[order]
        ens.set_inputs(torch.as_tensor(rm, dtype=torch.float64).to(device))
        ens.step_advance()
        for m, p in enumerate(plains):
            p.set_inputs(torch.as_tensor(np.ascontiguousarray(rm[:, m]), dtype=torch.float64).to(device))
            p.step_advance()
    torch.cuda.synchronize()
    a = ens.state_tensors()
    for m, p in enumerate(plains):
        b = p.state_tensors()
        for k in b:
            np.testing.assert_array_equal(a[k][..., m].cpu().numpy(), b[k].cpu().numpy(),
                                          err_msg=f"member {m} field {k}")
    ens.check_status()
