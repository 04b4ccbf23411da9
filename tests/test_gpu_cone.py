"""Cone CME volume insertion on the GPU (hc_level_insert_cone) against the
oracle, at both orders, through the C ABI.

Tolerance 1e-13 normwise per component (max|gpu - oracle| / max|oracle|):
the arithmetic per cell is the oracle's, but the device contracts a*b+c
into FMA and its cell-centre directions and <det A> come from double
rather than long double evaluations.  Cells changed and the mass statistic
(1e-12 relative: the device sums in a different fixed order) are compared
too, and cells outside the cloud must keep their bits.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc

INNER = 21.5 * 6.96e10
C_MP = 1.67262192e-24


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _wind(po, orc):
    init = po.HcInit()
    init.kind = 1
    init.rho0, init.p0, init.vr, init.b0, init.r_ref = 700 * C_MP, 1e-7, 400e5, 5e-3, INNER
    init.pulse_amp = 0.0
    return orc.init(init)


@pytest.mark.parametrize("order", [2, 4])
@pytest.mark.parametrize("seed", [1, 2])
def test_insert_cone_matches_oracle(oracle_lib, order, seed):
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(seed)
    n = 16
    kw = dict(nr=n, na=n, spatial_order=order, riemann_solver=2 if order == 4 else 1)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevel(po.make_params(**kw))
    spec = hc.ConeSpec.on_inner_boundary(INNER, lat_deg=rng.uniform(-30, 30), lon_deg=rng.uniform(-30, 30),
                                         half_angle_deg=rng.uniform(20, 60), apex_speed=rng.uniform(500, 2000),
                                         density=rng.uniform(2, 6) * 700 * C_MP)
    spec.reference_height += rng.uniform(0, 10)
    cone = hc.prepare_cone(spec, INNER)
    ocone = po.cone_prepare(po.HcConeSpec(**{k: getattr(spec, k) for k in po.CONE_SPEC_FIELDS}), INNER)
    ju0 = _wind(po, orc)
    ref = ju0.copy()
    rstats = orc.insert_cone(ocone, cone.insertion_time, ref)
    g = torch.from_numpy(ju0.copy()).cuda()
    gstats = shell.insert_cone(cone, cone.insertion_time, g, stats=True).cpu().numpy()
    got = g.cpu().numpy()
    err = rel_err_components(got.reshape(6, 8, -1), ref.reshape(6, 8, -1))
    assert err.max() < 1e-13, err
    outside = np.all(ref.reshape(6, 8, -1) == ju0.reshape(6, 8, -1), axis=1)[:, None, :].repeat(8, axis=1)
    assert np.array_equal(got.reshape(6, 8, -1)[outside], ju0.reshape(6, 8, -1)[outside])
    assert gstats[0] == rstats[0] and rstats[0] > 0
    assert gstats[1] == pytest.approx(rstats[1], rel=1e-12)


def test_insert_cone_without_stats_and_in_a_graph():
    """The stats-free launch equals the stats launch bit for bit, and the
    insertion replays from a captured CUDA graph."""
    _need_gpu()
    shell = hc.Shell(hc.Params(nr=24, na=16, spatial_order=4, riemann_solver=2))
    spec = hc.ConeSpec.on_inner_boundary(INNER, lat_deg=5.0, lon_deg=-10.0, half_angle_deg=35.0)
    cone = hc.prepare_cone(spec, INNER)
    base = shell.init(hc.InitSpec())
    a = base.clone()
    b = base.clone()
    shell.insert_cone(cone, cone.insertion_time, a, stats=True)
    shell.insert_cone(cone, cone.insertion_time, b)
    assert torch.equal(a, b)
    c = base.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            shell.insert_cone(cone, cone.insertion_time, c)
    torch.cuda.current_stream().wait_stream(s)
    c.copy_(base)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(c, a)


def test_inserted_cloud_steps():
    """A wind with an inserted 1500 km/s, 45 degree cloud stays valid over
    RK4 steps at the CFL time step, at both orders."""
    _need_gpu()
    for order in (2, 4):
        shell = hc.Shell(hc.Params(nr=24, na=24, spatial_order=order, riemann_solver=2 if order == 4 else 1))
        ju = shell.init(hc.InitSpec())
        spec = hc.ConeSpec.on_inner_boundary(INNER, half_angle_deg=45.0, apex_speed=1500.0)
        cone = hc.prepare_cone(spec, INNER)
        shell.insert_cone(cone, cone.insertion_time, ju)
        time = torch.full((1,), cone.insertion_time, dtype=torch.float64, device="cuda")
        shell.advance(ju, 10, time)
        assert shell.valid(ju), order
        assert math.isfinite(time.item())


def test_o4_step_with_cloud_matches_oracle(oracle_lib):
    """Stage preparation and one RK4 step of a level holding a sharp cloud
    that reaches the panel seams: the seam ghosts whose fourth-order
    interpolation is inadmissible fall back to their donor cell's average on
    both sides alike.  Tolerances as for smooth states (prepare 1e-12, one
    step 1e-12), since the fallback decisions sit far from their bounds."""
    _need_gpu()
    po = oracle_lib
    n = 16
    kw = dict(nr=n, na=n, spatial_order=4, riemann_solver=2, berta_fallback_type=0)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevelO4(po.make_params(**kw))
    base = po.OracleLevel(po.make_params(**kw))
    ju = _wind(po, base)
    spec = hc.ConeSpec.on_inner_boundary(INNER, lat_deg=30.0, lon_deg=30.0, half_angle_deg=60.0, apex_speed=2000.0,
                                         density=6 * 700 * C_MP)
    ocone = po.cone_prepare(po.HcConeSpec(**{k: getattr(spec, k) for k in po.CONE_SPEC_FIELDS}), INNER)
    base.insert_cone(ocone, ocone.insertion_time, ju)
    ref = orc.prepare(ju, 0.0)
    got = shell.prepare(torch.from_numpy(ju).cuda(), 0.0).cpu().numpy()
    err = rel_err_components(got.reshape(6, 8, -1), ref.reshape(6, 8, -1))
    assert err.max() < 1e-12, err
    dt = 0.3 / orc.inv_dt(ju)
    g = torch.from_numpy(ju.copy()).cuda()
    orc.rk4_step(ju, dt, 0.0)
    shell.rk4_step(g, dt, 0.0)
    assert shell.valid(g)
    err = rel_err_components(g.cpu().numpy().reshape(6, 8, -1), ju.reshape(6, 8, -1))
    assert err.max() < 1e-12, err


def _volume_event(t):
    from heliocubed_b200 import _native as N
    ev = N.HcCmeEvent()
    ev.insertion_time, ev.feeding_end, ev.boundary = t, t, 0
    return ev


@pytest.mark.parametrize("order", [2, 4])
def test_schedule_scales_the_cfl_step(oracle_lib, order):
    """With a schedule, every hc_level_advance_cfl step's dt is CFL /
    (rate / fraction(time)) for the rate of the step's initial state, the
    fraction from the oracle's restatement of the reference schedule
    (1e-14), and a fourth-order Roe context's steps land on the Rusanov
    window's end."""
    _need_gpu()
    po = oracle_lib
    n = 16
    kw = dict(nr=n, na=n, spatial_order=order, riemann_solver=2 if order == 4 else 1)
    sh = hc.Shell(hc.Params(**kw))
    ju = sh.init(hc.InitSpec())
    t0 = 1000.0
    ev = [_volume_event(t0 - 500.0), _volume_event(t0 + 300.0)]
    sh.set_cme_schedule(ev)
    oev = []
    for e in ev:
        o = po.HcCmeEvent()
        o.insertion_time, o.feeding_end, o.boundary = e.insertion_time, e.feeding_end, e.boundary
        oev.append(o)
    time = torch.full((1,), t0, dtype=torch.float64, device="cuda")
    dt = torch.zeros(1, dtype=torch.float64, device="cuda")
    ends = []
    for _ in range(6):
        rate = float(sh.inv_dt_max(ju).item())
        t = float(time.item())
        frac, end = po.cme_schedule(oev, t, 0.5 if order == 4 else 1.0)
        sh.advance(ju, 1, time, dt)
        expect = 0.4 / (rate / frac)
        if order == 4 and t < end - 1e-9 * max(1.0, abs(end)):
            expect = 0.4 / max(rate / frac, 0.4 / (end - t))
            ends.append(end)
        assert float(dt.item()) == pytest.approx(expect, rel=1e-14)
    assert sh.valid(ju)
    if order == 4:
        assert ends, "the steps never entered the Rusanov window"


@pytest.mark.parametrize("order", [2, 4])
def test_rusanov_window_runs_the_rusanov_operator(order):
    """Inside the window a Roe context's step equals, bit for bit, the same
    step of a Rusanov context with the same schedule; a fixed-dt step after
    it runs Roe again."""
    _need_gpu()
    n = 16
    roe = hc.Shell(hc.Params(nr=n, na=n, spatial_order=order, riemann_solver=2))
    rus = hc.Shell(hc.Params(nr=n, na=n, spatial_order=order, riemann_solver=1))
    ju0 = roe.init(hc.InitSpec())
    for sh in (roe, rus):
        sh.set_cme_schedule([_volume_event(0.0)])
    a, b = ju0.clone(), ju0.clone()
    ta = torch.zeros(1, dtype=torch.float64, device="cuda")
    tb = torch.zeros(1, dtype=torch.float64, device="cuda")
    roe.advance(a, 1, ta)
    rus.advance(b, 1, tb)
    torch.cuda.synchronize()
    assert float(ta.item()) < 600.0          # still inside the window
    assert torch.equal(ta, tb)
    assert torch.equal(a, b)
    # a fixed-dt step runs the context's own solver
    d1, d2 = ju0.clone(), ju0.clone()
    roe.rk4_step(d1, 30.0, 0.0)
    rus.rk4_step(d2, 30.0, 0.0)
    assert not torch.equal(d1, d2)
    # without a schedule the Roe context differs
    roe.set_cme_schedule([])
    c = ju0.clone()
    tc = torch.zeros(1, dtype=torch.float64, device="cuda")
    roe.advance(c, 1, tc)
    assert not torch.equal(c, a)


def _entering(hcmod):
    spec = hcmod.ConeSpec(lat_deg=10.0, lon_deg=-20.0, half_angle_deg=40.0, apex_speed=1000.0,
                          reference_height=21.5, reference_time=0.0, density=4 * 700 * C_MP, temperature=1.0e6)
    return spec


@pytest.mark.parametrize("limiter,solver", [(3, 1), (1, 2)])
def test_inlet_matches_oracle(oracle_lib, limiter, solver):
    """A cloud entering through the inner boundary of an order-2 level:
    the prepared primitives (inner-ghost inlet, 1e-13) and one RK4 step
    (ghost inlet every stage and the footprint of the inner faces, 1e-12)
    against the oracle."""
    _need_gpu()
    po = oracle_lib
    n = 16
    kw = dict(nr=n, na=n, spatial_order=2, limiter=limiter, riemann_solver=solver)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevel(po.make_params(**kw))
    spec = _entering(hc)
    cone = hc.prepare_cone(spec, INNER)
    ocone = po.cone_prepare(po.HcConeSpec(**{k: getattr(spec, k) for k in po.CONE_SPEC_FIELDS}), INNER)
    shell.set_inlet([cone])
    orc.set_inlet([ocone])
    ju = _wind(po, orc)
    t = 3000.0
    ref = orc.prepare(ju, t)
    got = shell.prepare(torch.from_numpy(ju).cuda(), t).cpu().numpy()
    w0 = orc.prepare(ju, 0.0)
    assert not np.array_equal(ref, w0)
    err = rel_err_components(got.reshape(6, 8, -1), ref.reshape(6, 8, -1))
    assert err.max() < 1e-13, err
    dt = 0.3 / orc.inv_dt(ju)
    g = torch.from_numpy(ju.copy()).cuda()
    ref_state = ju.copy()
    orc.rk4_step(ref_state, dt, t)
    shell.rk4_step(g, dt, t)
    assert shell.valid(g)
    err = rel_err_components(g.cpu().numpy().reshape(6, 8, -1), ref_state.reshape(6, 8, -1))
    assert err.max() < 1e-12, err
    # the inlet changed the step
    plain = ju.copy()
    orc.set_inlet([])
    orc.rk4_step(plain, dt, t)
    assert not np.array_equal(plain, ref_state)


@pytest.mark.parametrize("density_factor", [4.0, 0.25])
def test_inlet_adds_the_crossing_rate(oracle_lib, density_factor):
    """hc_level_advance_cfl with a crossing cloud: dt = CFL / (rate + (speed
    + sound speed) / first radial cell width), the rate's Alfven speeds
    taken with density min(rho, cone density) (the oracle's rate, 1e-13):
    a light cone raises the rate."""
    _need_gpu()
    po = oracle_lib
    n = 16
    p = hc.Params(nr=n, na=n)
    shell = hc.Shell(p)
    orc = po.OracleLevel(po.make_params(nr=n, na=n))
    spec = _entering(hc)
    spec.density = density_factor * 700 * C_MP
    cone = hc.prepare_cone(spec, INNER)
    ocone = po.cone_prepare(po.HcConeSpec(**{k: getattr(spec, k) for k in po.CONE_SPEC_FIELDS}), INNER)
    shell.set_inlet([cone])
    orc.set_inlet([ocone])
    ju0 = _wind(po, orc)
    ju = torch.from_numpy(ju0.copy()).cuda()
    time = torch.full((1,), 3000.0, dtype=torch.float64, device="cuda")
    dt = torch.zeros(1, dtype=torch.float64, device="cuda")
    rate = orc.inv_dt_at(ju0, 3000.0)
    plain = orc.inv_dt(ju0)
    assert (rate > plain * (1 + 1e-9)) == (density_factor < 1)
    shell.advance(ju, 1, time, dt)
    width = (p.outer_radius - p.inner_radius) * math.expm1(p.radial_stretch / n) / math.expm1(p.radial_stretch)
    boundary = (cone.speed * 1e5 + math.sqrt(p.gamma * 2 * 1.380649e-16 * cone.temperature / C_MP)) / width
    assert float(dt.item()) == pytest.approx(p.cfl / (rate + boundary), rel=1e-13)
    assert shell.valid(ju)
