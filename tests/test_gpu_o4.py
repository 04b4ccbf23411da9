"""Fourth-order Berta WENOZ operator (hc_box_rhs_o4) vs the oracle through
the C ABI, on single ghosted boxes (BertaOperator,
src/BoxOp_BertaCubedSphereImplem.H:1737-2076).

Tolerance: 1e-12 normwise per component for rhs and fluxes (gravity 1e-13) (the device
contracts a*b+c into FMA; the oracle does not).  Inputs are seeded:
a smooth wind (detector quiet) and a field with a sharp jump (detector
fires, WENO3 / PLM fallbacks and the Roe repair are exercised).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

C_MP = 1.67262192e-24
RS = 6.96e10


def usph_box(nr, lo, hi, g, seed=0, pert=0.05, jump=False):
    """Native conserved cell averages (point values of a seeded field) on
    valid.grow(g): Parker-like wind with angular perturbations; with
    jump=True a density/pressure step across the box."""
    rng = np.random.default_rng(seed)
    r0, r1, C = 21.5 * RS, 215 * RS, 1.5
    Rt = (r1 - r0) / np.expm1(C)
    glo = [lo[d] - g for d in range(3)]
    ghi = [hi[d] + g for d in range(3)]
    i = np.arange(glo[0], ghi[0] + 1)
    jj = np.arange(glo[1], ghi[1] + 1)
    kk = np.arange(glo[2], ghi[2] + 1)
    r = r0 + Rt * np.expm1(C * (i + 0.5) / nr)
    s = r0 / r
    ph = rng.uniform(0, 2 * np.pi, 4)
    ang = np.sin(0.3 * jj + ph[0])[None, :, None] * np.cos(0.2 * kk + ph[1])[:, None, None]
    rho = 700 * C_MP * s ** 2 * (1 + pert * ang)
    if jump:
        rho = rho * np.where((jj[None, :, None] + kk[:, None, None]) > (lo[1] + hi[1] + lo[2] + hi[2]) // 2, 3.0, 1.0)
    p = 1e-7 * s ** (10 / 3) * np.ones_like(rho)
    if jump:
        p = p * np.where(i[None, None, :] > (lo[0] + hi[0]) // 2, 2.5, 1.0)
    vr = 4e7
    U = np.zeros((8,) + rho.shape)
    U[0] = rho
    U[1] = rho * vr * (1 + 0.02 * ang)
    U[2] = rho * vr * 0.01 * np.cos(0.4 * jj + ph[2])[None, :, None]
    U[3] = rho * vr * 0.01 * ang
    U[5] = 5e-3 * s ** 2 * (1 + 0.1 * ang)
    U[6] = 1e-5 * ang * s
    U[7] = 2e-5 * np.cos(0.3 * kk + ph[3])[:, None, None] * s
    U[4] = p / (2 / 3) + 0.5 * rho * vr ** 2 + U[5] ** 2 / (8 * np.pi)
    return np.ascontiguousarray(U.reshape(-1))


CASES = [
    # riemann, fallback, jump, block, lo, hi
    (1, 0, False, 1, (3, 2, 4), (10, 9, 11)),
    (2, 0, False, 4, (0, 0, 5), (7, 6, 12)),
    (2, 0, True, 2, (2, 3, 1), (9, 10, 8)),
    (1, 1, True, 5, (4, 9, 0), (11, 15, 6)),
    (2, 1, True, 0, (0, 0, 0), (6, 7, 5)),
]


@pytest.mark.parametrize("riemann,fallback,jump,block,lo,hi", CASES)
def test_box_operator_o4_matches_oracle(oracle_lib, riemann, fallback, jump, block, lo, hi):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import make_box
    po = oracle_lib
    nr, na, g = 16, 16, 5
    kw = dict(nr=nr, na=na, spatial_order=4, riemann_solver=riemann, berta_fallback_type=fallback)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevel(po.make_params(**kw))
    u = usph_box(nr, lo, hi, g, seed=block, jump=jump)
    v = [hi[d] - lo[d] + 1 for d in range(3)]
    nv = v[0] * v[1] * v[2]
    rng = np.random.default_rng(3)
    rhs0 = rng.standard_normal(8 * nv) * 1e10
    fsz = [8 * (v[0] + (d == 0)) * (v[1] + (d == 1)) * (v[2] + (d == 2)) for d in range(3)]
    box_o = po.HcBox()
    for d in range(3):
        box_o.lo[d], box_o.hi[d] = lo[d], hi[d]
    box_o.ghost, box_o.block = g, block
    rhs_o = rhs0.copy()
    flux_o = [np.zeros(n) for n in fsz]
    orc.box_rhs_o4(box_o, u, rhs_o, flux_o, 0.5)
    assert np.isfinite(rhs_o).all()
    rhs_g = torch.from_numpy(rhs0.copy()).cuda()
    flux_g = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in fsz]
    shell.box_rhs_o4(make_box(lo, hi, g, block), torch.from_numpy(u).cuda(), rhs_g, flux_g, 0.5)
    torch.cuda.synchronize()
    err = rel_err_components(rhs_g.cpu().numpy().reshape(8, -1) - rhs0.reshape(8, -1),
                             rhs_o.reshape(8, -1) - rhs0.reshape(8, -1), 0)
    assert err.max() < 1e-12, err
    for d in range(3):
        e = rel_err_components(flux_g[d].cpu().numpy().reshape(8, -1), flux_o[d].reshape(8, -1), 0)
        assert e.max() < 1e-12, (d, e)
    shell.close()


@pytest.mark.parametrize("block,lo,hi,g", [(3, (2, 0, 5), (9, 6, 15), 5), (1, (0, 4, 0), (5, 15, 3), 1)])
def test_box_gravity_o4_matches_oracle(oracle_lib, block, lo, hi, g):
    """Gravity_Euler (src/BoxOp_Gravity.H:84-164) through hc_box_gravity_o4,
    boxes at panel edges (the angular metric products reach outside)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import make_box
    po = oracle_lib
    nr, na = 16, 16
    kw = dict(nr=nr, na=na, spatial_order=4, riemann_solver=2, sun_gravity=1)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevel(po.make_params(**kw))
    u = usph_box(nr, lo, hi, g, seed=block)
    v = [hi[d] - lo[d] + 1 for d in range(3)]
    rhs0 = np.random.default_rng(5).standard_normal(8 * v[0] * v[1] * v[2]) * 1e-3
    box_o = po.HcBox()
    for d in range(3):
        box_o.lo[d], box_o.hi[d] = lo[d], hi[d]
    box_o.ghost, box_o.block = g, block
    rhs_o = rhs0.copy()
    orc.box_gravity_o4(box_o, u, rhs_o)
    rhs_g = torch.from_numpy(rhs0.copy()).cuda()
    shell.box_gravity_o4(make_box(lo, hi, g, block), torch.from_numpy(u).cuda(), rhs_g)
    got = rhs_g.cpu().numpy().reshape(8, -1) - rhs0.reshape(8, -1)
    ref = rhs_o.reshape(8, -1) - rhs0.reshape(8, -1)
    assert np.abs(ref[[0, 5, 6, 7]]).max() == 0.0 and np.abs(got[[0, 5, 6, 7]]).max() == 0.0
    err = np.abs(got[[1, 2, 3, 4]] - ref[[1, 2, 3, 4]]).max(axis=1) / np.abs(ref[[1, 2, 3, 4]]).max(axis=1)
    assert err.max() < 1e-13, err
    shell.close()
