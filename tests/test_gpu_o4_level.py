"""Fourth-order level step, CUDA vs the oracle through the C ABI: stage
preparation (hc_level_prepare: Cartesian conversion, seam ghosts with panel
corners, native conversion, radial ghosts), the six-panel operator
(hc_level_rhs), RK4 steps with the seam flux register and reflux
(hc_level_rk4_step), the CFL rate (hc_level_dt_cfl) and the device-dt loop
(hc_level_advance_cfl).

Tolerances (FP64, normwise per component, max|gpu-oracle| / max|oracle|):
  prepare, one step        1e-12
  rhs                      5e-12 (the rhs is a difference of face fluxes
                           several orders larger than itself; its round-off
                           is relative to the fluxes, not to max|rhs|)
  CFL rate                 1e-13
  three steps, advance     1e-11
The device contracts a*b+c into FMA where the oracle does not.  States are
smooth (a seeded pulse plus smooth tangential flow and field), so the
detector and limiter switches do not sit on round-off.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc

PERM = [[1, 2, 0], [1, 2, 0], [1, 0, 2], [0, 1, 2], [1, 0, 2], [0, 1, 2]]
SIGN = [[1, -1, -1], [1, 1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1], [-1, -1, 1]]
GAMMA = 5.0 / 3.0

CASES = [
    dict(riemann_solver=2, berta_fallback_type=0, divergence_cleaning=1),
    dict(riemann_solver=1, berta_fallback_type=1, divergence_cleaning=1),
    dict(riemann_solver=2, berta_fallback_type=0, divergence_cleaning=1, sun_gravity=1),
]


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _unit(b, x1, x2):
    a = np.tan(-np.pi / 4 + np.pi / 2 * x1)
    c = np.tan(-np.pi / 4 + np.pi / 2 * x2)
    rho = np.sqrt(1 + a * a + c * c)
    q = [1 / rho, a / rho, c / rho]
    return np.array([SIGN[b][k] * q[PERM[b][k]] for k in range(3)])


def _pair(po, nr=16, na=16, **case):
    _need_gpu()
    kw = dict(nr=nr, na=na, spatial_order=4, sun_gravity=0)
    kw.update(case)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevelO4(po.make_params(**kw))
    return shell, orc


def _state(po, orc, seed=5):
    """Seeded pressure pulse on the analytic wind plus smooth tangential
    velocity (2 % of v_r) and field; pressure kept from the pulse state."""
    nr, na = orc.nr, orc.na
    spec = hc.InitSpec.seeded(seed, nr, na, margin=4)
    s = po.HcInit()
    s.kind = 1
    for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref", "pulse_amp",
              "pulse_width"):
        setattr(s, k, getattr(spec, k))
    ju = orc.init(s).reshape(6, 8, na, na, nr)
    det = orc.base.geometry(4).reshape(6, na, na)
    vol = orc.base.geometry(0).reshape(nr + 1, 4)[:nr, 3]
    J = det[:, :, :, None] * vol[None, None, None, :]
    rng = np.random.default_rng(seed)
    a, bv = rng.normal(size=3), rng.normal(size=3)
    x = (np.arange(na) + 0.5) / na
    for b in range(6):
        X = _unit(b, x[None, :], x[:, None])  # (3, k, j)
        pat = np.sin(a @ X.reshape(3, -1)).reshape(na, na)
        u = ju[b] / J[b][None]
        rho = u[0]
        m, B = u[1:4], u[5:8]
        p = (u[4] - 0.5 * (m ** 2).sum(0) / rho - (B ** 2).sum(0) / (8 * np.pi)) * (GAMMA - 1)
        vt = 8e5 * np.cross(a, X, axis=0)[:, :, :, None] * pat[None, :, :, None]
        bt = 1e-4 * np.cross(bv, X, axis=0)[:, :, :, None] * pat[None, :, :, None] * (vol[0] / vol)[None, None, None, :]
        m = m + rho[None] * vt
        B = B + bt
        u[1:4], u[5:8] = m, B
        u[4] = p / (GAMMA - 1) + 0.5 * (m ** 2).sum(0) / rho + (B ** 2).sum(0) / (8 * np.pi)
        ju[b] = u * J[b][None]
    return np.ascontiguousarray(ju.reshape(-1))


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _err(gpu, ref):
    return rel_err_components(np.asarray(gpu).reshape(6, 8, -1), np.asarray(ref).reshape(6, 8, -1))


@pytest.mark.parametrize("case", CASES)
def test_prepare_matches_oracle(oracle_lib, case):
    shell, orc = _pair(oracle_lib, **case)
    ju = _state(oracle_lib, orc)
    t = 3.0e4
    ref = orc.prepare(ju, t)
    got = shell.prepare(_t(ju), t).cpu().numpy()
    assert np.isfinite(got).all()
    assert _err(got, ref).max() < 1e-12, _err(got, ref)


@pytest.mark.parametrize("case", CASES)
def test_level_rhs_matches_oracle(oracle_lib, case):
    shell, orc = _pair(oracle_lib, **case)
    us = orc.prepare(_state(oracle_lib, orc), 0.0)
    ref = orc.rhs(us)
    got = shell.rhs(_t(us)).cpu().numpy()
    assert _err(got, ref).max() < 5e-12, _err(got, ref)


def test_cfl_rate_matches_oracle(oracle_lib):
    shell, orc = _pair(oracle_lib, **CASES[0])
    ju = _state(oracle_lib, orc)
    ref = orc.inv_dt(ju)
    got = float(shell.inv_dt_max(_t(ju)).item())
    assert abs(got - ref) <= 1e-13 * ref


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("nsteps", [1, 3])
def test_rk4_steps_match_oracle(oracle_lib, case, nsteps):
    shell, orc = _pair(oracle_lib, **case)
    ju = _state(oracle_lib, orc)
    dt = 0.3 / orc.inv_dt(ju)
    g = _t(ju)
    t = 1.0e3
    for n in range(nsteps):
        orc.rk4_step(ju, dt, t + n * dt)
        shell.rk4_step(g, dt, t + n * dt)
    got = g.cpu().numpy()
    tol = 1e-12 if nsteps == 1 else 1e-11
    assert np.isfinite(got).all()
    assert _err(got, ju).max() < tol, _err(got, ju)
    assert shell.valid(g)


def test_advance_cfl_matches_oracle(oracle_lib):
    shell, orc = _pair(oracle_lib, **CASES[0])
    ju = _state(oracle_lib, orc)
    g = _t(ju)
    time = torch.zeros(1, dtype=torch.float64, device="cuda")
    shell.advance(g, 2, time)
    t = 0.0
    for _ in range(2):
        dt = 0.4 / orc.inv_dt(ju)
        orc.rk4_step(ju, dt, t)
        t += dt
    assert abs(time.item() - t) <= 1e-12 * t
    assert _err(g.cpu().numpy(), ju).max() < 1e-11


def test_total_mass_matches_oracle(oracle_lib):
    """The level's total mass after one step (seam reflux included) agrees
    with the oracle's to round-off relative to the summed cell masses."""
    shell, orc = _pair(oracle_lib, **CASES[0])
    ju = _state(oracle_lib, orc)
    dt = 0.3 / orc.inv_dt(ju)
    g = _t(ju)
    shell.rk4_step(g, dt, 0.0)
    orc.rk4_step(ju, dt, 0.0)
    dm_gpu = g.cpu().numpy().reshape(6, 8, -1)[:, 0].sum()
    dm_ref = ju.reshape(6, 8, -1)[:, 0].sum()
    assert abs(dm_gpu - dm_ref) <= 1e-12 * abs(ju.reshape(6, 8, -1)[:, 0]).sum()
