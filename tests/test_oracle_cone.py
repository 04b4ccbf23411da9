"""Cone CME, finite spherical cloud (field model 4), on the CPU.

* The oracle's preparation (prepareConeCloud with the drag-based trajectory
  and the boundary-contact bisection) and its per-cell insertion increment
  are pinned bit-exactly against the reference's own src/MHD_CME.H compiled
  from source (oracle/_ref/libhcref.so; skipped where that was not built).
* The product library's host-side hc_cone_prepare equals the oracle
  bit-exactly and rejects the inputs it documents.
* The oracle's level insertion: cells outside the cloud keep their bits,
  cells inside take the cloud's density, radial speed and pressure
  2 k T rho / m_p with their field kept, and the mass statistic is the
  summed change of the density averages.
* The insertion schedule (CFL fraction, Rusanov window end) equals the
  reference's CMEInsertionSchedule bit for bit.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from oracle import pyoracle as po

INNER = 21.5 * 6.96e10
C_MP = 1.67262192e-24
K_B = 1.380649e-16


def _spec(rng, drag: bool, below: bool = False) -> po.HcConeSpec:
    s = po.HcConeSpec()
    s.lat_deg = rng.uniform(-30, 30)
    s.lon_deg = rng.uniform(-180, 180)
    s.half_angle_deg = rng.uniform(20, 60)
    s.apex_speed = rng.uniform(500, 2000)
    s.wind_speed = rng.uniform(300, 500)
    s.drag_gamma = rng.uniform(0.05e-7, 2e-7) if drag else 0.0
    s.reference_height = rng.uniform(10, 21) if below else rng.uniform(22, 80)
    s.reference_time = rng.uniform(-2e4, 2e4)
    s.density = rng.uniform(2, 6) * 700 * C_MP
    s.temperature = rng.uniform(5e5, 2e6)
    return s


def _cone_vec(c: po.HcCone) -> np.ndarray:
    return np.array([c.axis[0], c.axis[1], c.axis[2], c.radius, c.entry_shift, c.entry_time, c.speed,
                     c.end_time, c.insertion_time])


def _need_ref():
    if po.ref_lib() is None:
        pytest.skip("reference pin library not built (reference tree absent)")


@pytest.mark.parametrize("drag,below", [(False, False), (False, True), (True, False), (True, True)])
def test_prepare_matches_reference(drag, below):
    _need_ref()
    rng = np.random.default_rng(11 + 2 * drag + below)
    checked = 0
    for _ in range(40):
        s = _spec(rng, drag, below)
        ref = po.ref_cone_prepare(s, INNER)
        got = po.cone_prepare(s, INNER)
        assert (ref is None) == (got is None)
        if ref is None:
            continue
        np.testing.assert_array_equal(_cone_vec(got), ref)
        checked += 1
    assert checked >= 30


def test_prepare_slow_cone_in_fast_wind():
    """apex below the wind speed with drag: the branch with its own lower
    limit; success and failure agree with the reference."""
    _need_ref()
    rng = np.random.default_rng(5)
    for _ in range(40):
        s = _spec(rng, True)
        s.apex_speed = rng.uniform(200, 350)
        s.wind_speed = rng.uniform(400, 600)
        ref = po.ref_cone_prepare(s, INNER)
        got = po.cone_prepare(s, INNER)
        assert (ref is None) == (got is None)
        if ref is not None:
            np.testing.assert_array_equal(_cone_vec(got), ref)


def test_cell_increment_matches_reference():
    _need_ref()
    rng = np.random.default_rng(3)
    gamma = 5.0 / 3.0
    inside_count = 0
    for n in range(400):
        s = _spec(rng, n % 2 == 1)
        cone = po.cone_prepare(s, INNER)
        if cone is None:
            continue
        time = cone.insertion_time + rng.uniform(0, 3e3)
        shift = cone.entry_shift + cone.speed * 1e5 * (time - cone.entry_time)
        axis = np.array(cone.axis[:])
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        pos = shift * axis + cone.radius * rng.uniform(0, 1.3) * u
        amb = np.array([rng.uniform(1, 8) * 700 * C_MP * (21.5 * 6.96e10 / np.linalg.norm(pos)) ** 2,
                        *rng.normal(size=3) * 4e7, rng.uniform(0, 2e-7), *rng.normal(size=3) * 1e-3])
        if n % 7 == 0:
            amb[4] = 0.0
        ins_r, d_r = po.ref_cone_cell(s, INNER, time, pos, amb, gamma)
        ins_o, d_o = po.cone_cell(cone, time, pos, amb, gamma)
        assert ins_r == ins_o
        if ins_r:
            inside_count += 1
            np.testing.assert_array_equal(d_o, d_r)
    assert inside_count > 100


def test_library_prepare_matches_oracle():
    import heliocubed_b200 as hc
    from heliocubed_b200 import _native as N
    rng = np.random.default_rng(21)
    for n in range(30):
        s = _spec(rng, n % 2 == 1)
        ref = po.cone_prepare(s, INNER)
        spec = hc.ConeSpec(**{k: getattr(s, k) for k in po.CONE_SPEC_FIELDS})
        if ref is None:
            with pytest.raises(hc.HcError):
                hc.prepare_cone(spec, INNER)
            continue
        got = hc.prepare_cone(spec, INNER)
        np.testing.assert_array_equal(
            np.array([got.axis[0], got.axis[1], got.axis[2]] + [getattr(got, k) for k in N._CONE]),
            np.array([ref.axis[0], ref.axis[1], ref.axis[2]] + [getattr(ref, k) for k in po.CONE_FIELDS]))


@pytest.mark.parametrize("bad", [dict(drag_gamma=-1e-7), dict(half_angle_deg=0.0), dict(half_angle_deg=90.0),
                                 dict(apex_speed=0.0), dict(density=0.0)])
def test_library_prepare_rejects(bad):
    import heliocubed_b200 as hc
    with pytest.raises(hc.HcError):
        hc.prepare_cone(hc.ConeSpec(**bad), INNER)


def test_cloud_on_inner_boundary_is_inserted_whole():
    """A cloud whose leading edge sits at r_inner (1 + 2 sin a) at the
    reference time has its centre at r_inner + a then: the boundary never
    feeds it (end time = insertion time)."""
    import heliocubed_b200 as hc
    spec = hc.ConeSpec.on_inner_boundary(INNER, half_angle_deg=45.0, apex_speed=1500.0)
    cone = hc.prepare_cone(spec, INNER)
    a = INNER * math.sin(math.radians(45.0))
    assert cone.radius == pytest.approx(a, rel=1e-15)
    shift = cone.entry_shift + cone.speed * 1e5 * (cone.insertion_time - cone.entry_time)
    assert shift == pytest.approx(INNER + a, rel=1e-12)
    assert cone.end_time == pytest.approx(cone.insertion_time, rel=1e-12, abs=1e-6)


def test_level_insertion_properties():
    params = po.make_params(nr=12, na=12)
    orc = po.OracleLevel(params)
    init = po.HcInit()
    init.kind = 1
    init.rho0, init.p0, init.vr, init.b0, init.r_ref = 700 * C_MP, 1e-7, 400e5, 5e-3, INNER
    ju0 = orc.init(init)
    s = po.HcConeSpec()
    s.lat_deg, s.lon_deg, s.half_angle_deg = 10.0, 20.0, 40.0
    s.apex_speed, s.wind_speed, s.drag_gamma = 1500.0, 400.0, 0.0
    s.reference_height = 21.5 * (1 + 2 * math.sin(math.radians(40.0))) + 5.0
    s.reference_time, s.density, s.temperature = 0.0, 4 * 700 * C_MP, 1.0e6
    cone = po.cone_prepare(s, INNER)
    ju = ju0.copy()
    stats = orc.insert_cone(cone, cone.insertion_time, ju)
    a = ju0.reshape(6, 8, -1)
    b = ju.reshape(6, 8, -1)
    changed = np.any(a != b, axis=1)
    assert stats[0] == changed.sum() and stats[0] > 20
    det = orc.L.orc_geometry  # geometry export of the oracle level
    nr, na = 12, 12
    detv = np.zeros(6 * na * na)
    det(orc.h, 4, po.dptr(detv))
    rad = np.zeros((nr + 1) * 4)
    det(orc.h, 0, po.dptr(rad))
    J = (detv.reshape(6, na, na)[:, :, :, None] * rad.reshape(nr + 1, 4)[:nr, 3][None, None, None, :]).reshape(6, -1)
    u = b / J[:, None, :]
    rho = u[:, 0][changed]
    assert np.allclose(rho, s.density, rtol=1e-14, atol=0)
    v = u[:, 1:4] / u[:, 0:1]
    speed = np.sqrt((v ** 2).sum(1))[changed]
    assert np.allclose(speed, cone.speed * 1e5, rtol=1e-13)
    Bf = u[:, 5:8]
    np.testing.assert_array_equal(b[:, 5:8], a[:, 5:8])
    p = (u[:, 4] - 0.5 * u[:, 0] * (v ** 2).sum(1) - (Bf ** 2).sum(1) / (8 * np.pi)) * (2.0 / 3.0)
    assert np.allclose(p[changed], 2 * K_B * s.temperature * s.density / C_MP, rtol=1e-9)
    dm = ((b[:, 0] - a[:, 0]) / nr / na / na).sum()
    assert stats[1] == pytest.approx(dm, rel=1e-12)
    # a second insertion at the same time leaves the state within round-off
    again = ju.copy()
    orc.insert_cone(cone, cone.insertion_time, again)
    assert np.abs(again - ju).max() <= 1e-13 * np.abs(ju).max()


def _events(times, ends):
    out = []
    for t, e in zip(times, ends):
        ev = po.HcCmeEvent()
        ev.insertion_time = t
        ev.boundary = 1 if e > t else 0
        ev.feeding_end = max(t, e)
        out.append(ev)
    return out


@pytest.mark.parametrize("feeding", [0.5, 1.0])
def test_cme_schedule_matches_reference(feeding):
    """The oracle's CFL fraction and Rusanov window end equal the reference's
    CMEInsertionSchedule (compiled from src/MHD_CME.H) bit for bit: volume
    and boundary sources, before, inside and after their windows."""
    _need_ref()
    rng = np.random.default_rng(int(feeding * 10))
    for _ in range(30):
        n = int(rng.integers(1, 5))
        times = np.sort(rng.uniform(0, 2e4, n))
        ends = times + np.where(rng.random(n) < 0.5, rng.uniform(-500, 0, n), rng.uniform(10, 5000, n))
        events = _events(times, ends)
        for time in rng.uniform(-100, 3e4, 12):
            inserted = int((times <= time).sum())
            ref = po.ref_cme_schedule(times, ends, inserted, time, 1.0, feeding)
            got = po.cme_schedule(events, time, feeding)
            assert got[0] == ref[0], (time, got, ref)
            if inserted:
                assert got[1] == ref[1]


def test_library_cone_event_matches_schedule_rule():
    """hc_cone_event marks a cone as a boundary source exactly when its
    cloud ends after insertion (src/MHD_CME.H:1251-1253)."""
    import heliocubed_b200 as hc
    from heliocubed_b200 import _native as N
    lib = N.lib()
    for spec in (hc.ConeSpec.on_inner_boundary(INNER, half_angle_deg=30.0),
                 hc.ConeSpec(reference_height=21.5, half_angle_deg=30.0, apex_speed=1000.0)):
        cone = hc.prepare_cone(spec, INNER)
        ev = N.HcCmeEvent()
        assert lib.hc_cone_event(C.byref(cone), C.byref(ev)) == 0
        assert ev.boundary == (1 if cone.end_time > cone.insertion_time else 0)
        assert ev.feeding_end == max(cone.insertion_time, cone.end_time)


def _entering_cone(t_ref=0.0):
    s = po.HcConeSpec()
    s.lat_deg, s.lon_deg, s.half_angle_deg = 10.0, -20.0, 40.0
    s.apex_speed, s.wind_speed, s.drag_gamma = 1000.0, 400.0, 0.0
    s.reference_height, s.reference_time = 21.5, t_ref      # leading edge on r_inner: entering now
    s.density, s.temperature = 4 * 700 * C_MP, 1.0e6
    return po.cone_prepare(s, INNER)


def test_inlet_prescribes_the_cloud_in_inner_ghosts():
    """The oracle's inner ghosts under an entering cloud carry the cloud's
    density, radial speed and pressure with the wind's field; ghosts outside
    it keep the wind; without the inlet nothing changes."""
    nr, na = 12, 12
    params = po.make_params(nr=nr, na=na)
    orc = po.OracleLevel(params)
    init = po.HcInit()
    init.kind = 1
    init.rho0, init.p0, init.vr, init.b0, init.r_ref = 700 * C_MP, 1e-7, 400e5, 5e-3, INNER
    ju = orc.init(init)
    cone = _entering_cone()
    assert cone.insertion_time <= 0.0 < cone.end_time
    t = 3000.0
    base = orc.prepare(ju, t).reshape(6, 8, na + 4, na + 4, nr + 4)
    orc.set_inlet([cone])
    got = orc.prepare(ju, t).reshape(6, 8, na + 4, na + 4, nr + 4)
    ghosts = (slice(None), slice(None), slice(2, na + 2), slice(2, na + 2), slice(0, 2))
    changed = np.any(got[ghosts] != base[ghosts], axis=1)
    assert changed.sum() > 4
    g, b = got[ghosts], base[ghosts]
    assert np.allclose(g[:, 0][changed], cone.density, rtol=1e-13)
    speed = np.sqrt((g[:, 1:4] ** 2).sum(1))[changed]
    assert np.allclose(speed, cone.speed * 1e5, rtol=1e-12)
    assert np.allclose(g[:, 4][changed], 2 * K_B * cone.temperature * cone.density / C_MP, rtol=1e-10)
    assert np.allclose(np.moveaxis(g[:, 5:8], 1, -1)[changed], np.moveaxis(b[:, 5:8], 1, -1)[changed], rtol=1e-12,
                       atol=1e-30)
    # everything but the inner ghosts is untouched
    inner = np.zeros(got.shape, bool)
    inner[ghosts] = True
    assert np.array_equal(got[~inner], base[~inner])
    orc.set_inlet([])
    assert np.array_equal(orc.prepare(ju, t), base.reshape(-1))
