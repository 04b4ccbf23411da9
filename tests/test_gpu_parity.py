"""CUDA path vs the oracle, through the C ABI (libhc_b200.so).

Tolerances (FP64, normwise per component, max|gpu-oracle| / max|oracle|):
  pointwise conversions, geometry, CFL      1e-13
  operator rhs / fluxes on identical inputs 1e-12
  one RK4 step                              1e-12
  10 RK4 steps                              1e-10
The device code contracts a*b+c into FMA where the oracle (built with
-ffp-contract=off) does not, so agreement is to round-off, not bit-exact.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import make_box


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _params(**kw):
    p = dict(nr=12, na=10, limiter=3, riemann_solver=1, sun_gravity=1)
    p.update(kw)
    return p


def _pair(oracle_lib, **kw):
    _need_gpu()
    kw = _params(**kw)
    shell = hc.Shell(hc.Params(**kw))
    orc = oracle_lib.OracleLevel(oracle_lib.make_params(**kw))
    return shell, orc


def _spec(nr, na, seed=1):
    return hc.InitSpec.seeded(seed, nr, na, margin=2)


def _to_c_init(po, spec):
    s = po.HcInit()
    s.kind = 1
    for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref", "pulse_amp",
              "pulse_width"):
        setattr(s, k, getattr(spec, k))
    return s


def _perturbed_state(oracle_lib, orc, spec, seed=3, amp=0.05):
    """Oracle initial state with seeded multiplicative noise on every
    component (tangential velocity and field become nonzero)."""
    ju = orc.init(_to_c_init(oracle_lib, spec))
    rng = np.random.default_rng(seed)
    nr, na = orc.params.nr, orc.params.na
    v = ju.reshape(6, 8, na, na, nr)
    scale = np.abs(v).max(axis=(0, 2, 3, 4))
    # add tangential momentum / field of a few percent of the radial ones
    v[:, 1:4] += amp * scale[1:4, None, None, None] * rng.standard_normal(v[:, 1:4].shape) * 0.3
    v[:, 5:8] += amp * scale[5:8, None, None, None] * rng.standard_normal(v[:, 5:8].shape) * 0.3
    v[:, 4] *= 1 + amp * rng.random(v[:, 4].shape)
    return np.ascontiguousarray(v.reshape(-1))


def _used_mask(nr, na, g=2):
    """Cells of a ghosted level primitive array that the operator reads:
    valid cells, angular ghosts at valid radial/other-angular index, radial
    ghosts at valid angular indices (panel corners are never read)."""
    m = np.zeros((na + 2 * g, na + 2 * g, nr + 2 * g), dtype=bool)  # [k][j][i]
    vi, vj, vk = slice(g, g + nr), slice(g, g + na), slice(g, g + na)
    m[vk, vj, :] = True
    m[vk, :, vi] = True
    m[:, vj, vi] = True
    return m


def test_init_matches_oracle(oracle_lib):
    shell, orc = _pair(oracle_lib)
    spec = _spec(12, 10)
    ju_g = shell.init(spec).cpu().numpy()
    ju_o = orc.init(_to_c_init(oracle_lib, spec))
    err = rel_err_components(ju_g.reshape(6, 8, -1), ju_o.reshape(6, 8, -1))
    assert err.max() < 1e-13, err


def test_geometry_matches_oracle(oracle_lib):
    shell, orc = _pair(oracle_lib)
    for what in range(6):
        a, b = shell.geometry(what), orc.geometry(what)
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max(), what


@pytest.mark.parametrize("riemann", [1, 2])
def test_prepare_matches_oracle(oracle_lib, riemann):
    shell, orc = _pair(oracle_lib, riemann_solver=riemann)
    nr, na = 12, 10
    ju = _perturbed_state(oracle_lib, orc, _spec(nr, na))
    w_o = orc.prepare(ju, 0.0).reshape(6, 8, na + 4, na + 4, nr + 4)
    w_g = shell.prepare(torch.from_numpy(ju).cuda(), 0.0).cpu().numpy().reshape(6, 8, na + 4, na + 4, nr + 4)
    m = _used_mask(nr, na)
    err = rel_err_components(w_g[:, :, m], w_o[:, :, m])
    assert err.max() < 1e-13, err


@pytest.mark.parametrize("limiter,riemann", [(0, 1), (1, 1), (3, 1), (3, 2), (1, 2)])
def test_level_rhs_matches_oracle(oracle_lib, limiter, riemann):
    shell, orc = _pair(oracle_lib, limiter=limiter, riemann_solver=riemann)
    nr, na = 12, 10
    ju = _perturbed_state(oracle_lib, orc, _spec(nr, na, seed=limiter + 5))
    w = orc.prepare(ju, 0.0)
    k_o = orc.rhs(w)
    k_g = shell.rhs(torch.from_numpy(w).cuda()).cpu().numpy()
    err = rel_err_components(k_g.reshape(6, 8, -1), k_o.reshape(6, 8, -1))
    assert err.max() < 1e-12, err


@pytest.mark.parametrize("ghost,riemann", [(2, 1), (3, 2)])
def test_box_operator_matches_oracle(oracle_lib, ghost, riemann):
    """hc_box_rhs on an interior box with caller-owned rhs accumulation,
    flux outputs and adjacent-panel face states."""
    shell, orc = _pair(oracle_lib, riemann_solver=riemann)
    nr, na = 12, 10
    ju = _perturbed_state(oracle_lib, orc, _spec(nr, na, seed=11))
    w = orc.prepare(ju, 0.0).reshape(6, 8, na + 4, na + 4, nr + 4)
    block, lo, hi = 2, (3, 1, 2), (9, 8, 6)
    g = ghost
    # box storage valid.grow(g); level arrays carry 2 ghosts, so for g = 3
    # pad the stored primitive with an extra (never read) layer.
    wl = np.zeros((8, hi[2] - lo[2] + 1 + 2 * g, hi[1] - lo[1] + 1 + 2 * g, hi[0] - lo[0] + 1 + 2 * g))
    for k in range(wl.shape[1]):
        for j in range(wl.shape[2]):
            for i in range(wl.shape[3]):
                gk, gj, gi = lo[2] - g + k + 2, lo[1] - g + j + 2, lo[0] - g + i + 2
                if 0 <= gk < na + 4 and 0 <= gj < na + 4 and 0 <= gi < nr + 4:
                    wl[:, k, j, i] = w[block, :, gk, gj, gi]
    wl = np.ascontiguousarray(wl.reshape(-1))
    v = [hi[d] - lo[d] + 1 for d in range(3)]
    nv = v[0] * v[1] * v[2]
    rng = np.random.default_rng(5)
    rhs0 = rng.standard_normal(8 * nv) * 1e3
    fsz = [8 * (v[0] + (d == 0)) * (v[1] + (d == 1)) * (v[2] + (d == 2)) for d in range(3)]
    # adjacent-panel states on the low xi1 and high xi2 seam slabs
    slab1 = np.ascontiguousarray(np.repeat(w[block, :, lo[2] + 2:hi[2] + 3, lo[1] + 2, lo[0] + 2:hi[0] + 3][:, :, None, :],
                                           1, axis=2).reshape(-1) * (1 + 1e-3))
    slab2 = np.ascontiguousarray(w[block, :, hi[2] + 2, lo[1] + 2:hi[1] + 3, lo[0] + 2:hi[0] + 3].reshape(-1) * (1 - 1e-3))
    panel_o = [None, None, slab1, None, None, slab2]
    box_o = oracle_lib.HcBox()
    for d in range(3):
        box_o.lo[d], box_o.hi[d] = lo[d], hi[d]
    box_o.ghost, box_o.block = g, block
    rhs_o = rhs0.copy()
    flux_o = [np.zeros(n) for n in fsz]
    orc.box_rhs(box_o, wl, rhs_o, flux_o, panel_o, 0.75)
    box_g = make_box(lo, hi, g, block)
    rhs_g = torch.from_numpy(rhs0.copy()).cuda()
    flux_g = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in fsz]
    panel_g = [None if p is None else torch.from_numpy(p).cuda() for p in panel_o]
    shell.box_rhs(box_g, torch.from_numpy(wl).cuda(), rhs_g, flux_g, panel_g, 0.75)
    err = rel_err_components(rhs_g.cpu().numpy().reshape(8, -1), rhs_o.reshape(8, -1), 0)
    assert err.max() < 1e-12, err
    for d in range(3):
        e = rel_err_components(flux_g[d].cpu().numpy().reshape(8, -1), flux_o[d].reshape(8, -1), 0)
        assert e.max() < 1e-12, (d, e)
    # gravity on the same box
    rg_o = rhs0.copy()
    orc.box_gravity(box_o, wl, rg_o)
    rg_g = torch.from_numpy(rhs0.copy()).cuda()
    shell.box_gravity(box_g, torch.from_numpy(wl).cuda(), rg_g)
    assert np.abs(rg_g.cpu().numpy() - rg_o).max() <= 1e-13 * np.abs(rg_o).max()


def test_cfl_matches_oracle(oracle_lib):
    shell, orc = _pair(oracle_lib)
    ju = _perturbed_state(oracle_lib, orc, _spec(12, 10))
    a = shell.inv_dt_max(torch.from_numpy(ju).cuda()).item()
    b = orc.inv_dt(ju)
    assert abs(a - b) <= 1e-13 * b


@pytest.mark.parametrize("riemann", [1, 2])
def test_rk4_steps_match_oracle(oracle_lib, riemann):
    shell, orc = _pair(oracle_lib, riemann_solver=riemann)
    nr, na = 12, 10
    ju = _perturbed_state(oracle_lib, orc, _spec(nr, na, seed=riemann))
    dt = 0.4 / orc.inv_dt(ju)
    ju_o = ju.copy()
    ju_g = torch.from_numpy(ju.copy()).cuda()
    orc.rk4_step(ju_o, dt, 0.0)
    shell.rk4_step(ju_g, dt, 0.0)
    err = rel_err_components(ju_g.cpu().numpy().reshape(6, 8, -1), ju_o.reshape(6, 8, -1))
    assert err.max() < 1e-12, err
    for n in range(1, 10):
        orc.rk4_step(ju_o, dt, n * dt)
        shell.rk4_step(ju_g, dt, n * dt)
    err = rel_err_components(ju_g.cpu().numpy().reshape(6, 8, -1), ju_o.reshape(6, 8, -1))
    assert err.max() < 1e-10, err
    assert shell.valid(ju_g) and orc.valid(ju_o)


def test_advance_cfl_on_device(oracle_lib):
    """Device dt = cfl / max rate, steps chained without host sync."""
    shell, orc = _pair(oracle_lib)
    ju = _perturbed_state(oracle_lib, orc, _spec(12, 10))
    ju_o = ju.copy()
    t_o = 0.0
    for _ in range(3):
        dt = 0.4 / orc.inv_dt(ju_o)
        orc.rk4_step(ju_o, dt, t_o)
        t_o += dt
    ju_g = torch.from_numpy(ju.copy()).cuda()
    time = torch.zeros(1, dtype=torch.float64, device="cuda")
    shell.advance(ju_g, 3, time)
    assert abs(time.item() - t_o) <= 1e-12 * t_o
    err = rel_err_components(ju_g.cpu().numpy().reshape(6, 8, -1), ju_o.reshape(6, 8, -1))
    assert err.max() < 1e-11, err


def test_valid_flags_bad_cells(oracle_lib):
    shell, orc = _pair(oracle_lib)
    ju = _perturbed_state(oracle_lib, orc, _spec(12, 10))
    g = torch.from_numpy(ju.copy()).cuda()
    assert shell.valid(g) and orc.valid(ju)
    bad = ju.copy()
    bad[17] = np.nan
    assert not shell.valid(torch.from_numpy(bad).cuda()) and not orc.valid(bad)
    bad = ju.copy()
    bad[5] = -bad[5]   # negative density in panel 0
    assert not shell.valid(torch.from_numpy(bad).cuda()) and not orc.valid(bad)
    bad = ju.copy()
    bad[8 * 12 * 100 + 3] = np.inf  # energy... any component non-finite
    assert not shell.valid(torch.from_numpy(bad).cuda()) and not orc.valid(bad)


def test_seam_fluxes_conserve_mass(oracle_lib):
    """Total mass rhs equals the net radial boundary flux: panel-seam
    fluxes cancel because both panels solve the same shared-state problem."""
    shell, orc = _pair(oracle_lib, sun_gravity=0)
    nr, na = 12, 10
    ju = _perturbed_state(oracle_lib, orc, _spec(nr, na))
    w = shell.prepare(torch.from_numpy(ju).cuda())
    k = shell.rhs(w).cpu().numpy().reshape(6, 8, na, na, nr)
    total = k[:, 0].sum()
    # radial boundary fluxes through the per-box operator (dir 0 only)
    wv = w.cpu().numpy().reshape(6, 8, na + 4, na + 4, nr + 4)
    net = 0.0
    mag = 0.0
    for b in range(6):
        box = make_box((0, 0, 0), (nr - 1, na - 1, na - 1), 2, b)
        rhs = torch.zeros(8 * nr * na * na, dtype=torch.float64, device="cuda")
        f0 = torch.zeros(8 * (nr + 1) * na * na, dtype=torch.float64, device="cuda")
        shell.box_rhs(box, torch.from_numpy(np.ascontiguousarray(wv[b].reshape(-1))).cuda(), rhs, [f0, None, None])
        F = f0.cpu().numpy().reshape(8, na, na, nr + 1)[0]
        net += -nr * (F[:, :, nr].sum() - F[:, :, 0].sum())
        mag += nr * (np.abs(F[:, :, nr]).sum() + np.abs(F[:, :, 0]).sum())
    assert abs(total - net) <= 1e-12 * mag, (total, net, mag)


def test_graph_replay_matches_eager(oracle_lib):
    """The step captured as a CUDA graph replays the same launches."""
    shell, orc = _pair(oracle_lib)
    ju = _perturbed_state(oracle_lib, orc, _spec(12, 10))
    a = torch.from_numpy(ju.copy()).cuda()
    b = torch.from_numpy(ju.copy()).cuda()
    ta = torch.zeros(1, dtype=torch.float64, device="cuda")
    tb = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = shell.capture_advance(b, 1, tb)   # one eager step + capture
    shell.advance(a, 1, ta)
    for _ in range(3):
        g.replay()
        shell.advance(a, 1, ta)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(ta, tb)
