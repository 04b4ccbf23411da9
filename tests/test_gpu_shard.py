"""Radial slabs of one shell on the device path (heliocubed_b200.shard).

* hc_level_rk4_stage: stages 0..3 in order are hc_level_rk4_step, bit for
  bit, at both orders.
* Two and three slabs of one shell, all driven on one GPU in one process
  (halo layers moved by device copies between the slabs' buffers; nothing
  waits on another launch), step exactly like the whole shell: three RK4
  steps with the shell's CFL dt give bit-identical owned cells and the same
  CFL rates, at order 2 (PLM-MC with Rusanov and gravity, with Roe) and
  order 4 (Berta WENOZ + Roe with gravity).  With dt kept on the device
  (`advance`) the slabs equal the whole shell driven by the same code.
* A slab refuses the CME schedule and the boundary inlet (both steer the
  whole shell's dt) and a slab outside its shell."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200 import level as hl
    from heliocubed_b200 import _native as N
    from heliocubed_b200.shard import ShardedShell

CASES = {
    "o2_rusanov_gravity": dict(nr=32, na=16, spatial_order=2, limiter=3, riemann_solver=1, sun_gravity=1),
    "o2_roe": dict(nr=32, na=16, spatial_order=2, limiter=3, riemann_solver=2),
    "o4_roe_gravity": dict(nr=36, na=16, spatial_order=4, riemann_solver=2, sun_gravity=1, berta_fallback_type=0),
}


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _state(shell, p):
    det = shell.geometry(4).reshape(6, p.na, p.na)
    vol = shell.geometry(0).reshape(p.nr + 1, 4)[:p.nr, 3]
    return torch.from_numpy(np.ascontiguousarray(hl.perturbed_wind_state(p, det, vol, seed=5).reshape(-1))).cuda()


@pytest.mark.parametrize("case", sorted(CASES))
def test_stages_in_order_are_the_step(case):
    _need_gpu()
    p = hl.Params(**CASES[case])
    shell = hc.Shell(p)
    ju0 = _state(shell, p)
    a, b = ju0.clone(), ju0.clone()
    dt = p.cfl / float(shell.inv_dt_max(a)[0])
    for _ in range(2):
        shell.rk4_step(a, dt, 0.0)
        for s in range(4):
            shell.rk4_stage(b, s, dt, 0.0)
    torch.cuda.synchronize()
    assert torch.isfinite(a).all() and not torch.equal(a, ju0)
    assert torch.equal(a, b)
    shell.close()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", sorted(CASES))
def test_slabs_step_like_the_whole_shell(case, world):
    _need_gpu()
    p = hl.Params(**CASES[case])
    shell = hc.Shell(p)
    ju = _state(shell, p)
    sh = ShardedShell.emulated(p, world)
    states = sh.scatter(ju)
    for _ in range(3):
        inv_w = shell.inv_dt_max(ju)
        inv_s = sh.inv_dt_max(states)
        assert torch.equal(inv_w, inv_s)
        dt = p.cfl / float(inv_w[0])
        shell.rk4_step(ju, dt, 0.0)
        sh.rk4_step(states, dt, 0.0)
    torch.cuda.synchronize()
    got = sh.gather(states)
    want = ju.view(6, 8, p.na, p.na, p.nr)
    assert torch.isfinite(want).all()
    assert torch.equal(got, want), (got - want).abs().max().item()
    sh.close()
    shell.close()


@pytest.mark.parametrize("case", ["o2_roe", "o4_roe_gravity"])
def test_slabs_advance_with_device_dt(case):
    _need_gpu()
    p = hl.Params(**CASES[case])
    whole = ShardedShell.emulated(p, 1)
    ju = _state(whole.levels[0], p)
    sw = whole.scatter(ju)
    sh = ShardedShell.emulated(p, 3)
    ss = sh.scatter(ju)
    tw = torch.zeros(1, dtype=torch.float64, device="cuda")
    ts = torch.zeros(1, dtype=torch.float64, device="cuda")
    whole.advance(sw, 3, tw)
    sh.advance(ss, 3, ts)
    torch.cuda.synchronize()
    assert float(tw[0]) > 0 and torch.equal(tw, ts)
    assert torch.equal(sh.gather(ss), whole.gather(sw))
    sh.close()
    whole.close()


def test_slab_refusals():
    _need_gpu()
    base = dict(nr=12, na=16, spatial_order=2, radial_cells=40)
    with pytest.raises(N.HcError):
        hc.Shell(hl.Params(radial_offset=30, **base))           # beyond the shell
    with pytest.raises(N.HcError):
        hc.Shell(hl.Params(nr=12, na=16, radial_offset=3))      # an offset without a shell
    slab = hc.Shell(hl.Params(radial_offset=10, **base))
    spec = hl.ConeSpec.on_inner_boundary(slab.params.inner_radius)
    cone = hl.prepare_cone(spec, slab.params.inner_radius)
    with pytest.raises(N.HcError):
        slab.set_inlet([cone])
    ev = N.HcCmeEvent()
    ev.insertion_time, ev.feeding_end = 0.0, 1.0
    with pytest.raises(N.HcError):
        slab.set_cme_schedule([ev])
    slab.close()


def test_radial_window_limits_the_operator():
    """After stage 0 the next stage state is ju + (dt/2) k: with the window
    [lo, hi) it equals the whole level's inside the window and ju outside."""
    _need_gpu()
    p = hl.Params(**CASES["o4_roe_gravity"])
    full, win = hc.Shell(p), hc.Shell(p)
    lo, hi = 7, 23
    win.set_radial_window(lo, hi)
    ju = _state(full, p)
    dt = p.cfl / float(full.inv_dt_max(ju)[0])
    a, b = ju.clone(), ju.clone()
    full.rk4_stage(a, 0, dt, 0.0)
    win.rk4_stage(b, 0, dt, 0.0)
    sa = full.stage_state(a, 1)[0].view(6, 8, p.na, p.na, p.nr)
    sb = win.stage_state(b, 1)[0].view(6, 8, p.na, p.na, p.nr)
    u = ju.view(6, 8, p.na, p.na, p.nr)
    torch.cuda.synchronize()
    assert torch.equal(sb[..., lo:hi], sa[..., lo:hi])
    assert torch.equal(sb[..., :lo], u[..., :lo]) and torch.equal(sb[..., hi:], u[..., hi:])
    assert not torch.equal(sa[..., :lo], u[..., :lo])
    win.set_radial_window(0, 0)                               # the whole level again
    c = ju.clone()
    win.rk4_stage(c, 0, dt, 0.0)
    torch.cuda.synchronize()
    assert torch.equal(win.stage_state(c, 1)[0], full.stage_state(a, 1)[0])
    with pytest.raises(N.HcError):
        win.set_radial_window(5, 40)
    o2 = hc.Shell(hl.Params(**CASES["o2_roe"]))
    with pytest.raises(N.HcError):
        o2.set_radial_window(2, 10)
    for s in (full, win, o2):
        s.close()


def test_slab_admission_is_the_shells():
    """The served input (the wind with a cone cloud inserted on the device)
    built on each slab is that slab's part of the whole shell's, bit for
    bit, and the slabs then step like the shell."""
    _need_gpu()
    from heliocubed_b200 import serve
    p = hl.Params(**CASES["o4_roe_gravity"])
    shell = hc.Shell(p)
    cone = serve.Cone(speed_kms=1500.0, half_width_deg=45.0, lat_deg=10.0, lon_deg=-20.0, density_ratio=4.0)
    req = serve.Request(0, p.nr, p.na, 4, 1, 0.0, cone)
    ju = shell.new_state()
    t = torch.zeros(1, dtype=torch.float64, device="cuda")
    serve.admit(shell, req, ju, t, schedule=False)
    sh = ShardedShell.emulated(p, 3)
    states = []
    for lvl in sh.levels:
        st = lvl.new_state()
        serve.admit(lvl, req, st, torch.zeros(1, dtype=torch.float64, device="cuda"), schedule=False)
        states.append(st)
    torch.cuda.synchronize()
    full = ju.view(6, 8, p.na, p.na, p.nr)
    for plan, st in zip(sh.plans, states):
        assert torch.equal(st.view(6, 8, p.na, p.na, plan.local_nr), full[..., plan.offset:plan.offset + plan.local_nr])
    assert not torch.equal(ju, shell.init(serve.wind_spec()))       # the cloud is in
    dt = p.cfl / float(shell.inv_dt_max(ju)[0])
    shell.rk4_step(ju, dt, float(t[0]))
    sh.rk4_step(states, dt, float(t[0]))
    torch.cuda.synchronize()
    assert torch.equal(sh.gather(states), ju.view(6, 8, p.na, p.na, p.nr))
    sh.close()
    shell.close()
