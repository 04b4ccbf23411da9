"""Uniform-state preservation on the cubed sphere (the analytic check the
reference's metric design targets, src/BoxOp_SecondOrder.H:152-154 and
src/BoxOp_EulerCubedSphereImplem.H:21-25), on the device path.

* Second order (hc_box_rhs, PLM-MC with Rusanov and Roe, Powell): a uniform
  Cartesian state, at rest and moving, has zero flux divergence to
  round-off: |rhs| <= 1e-12 x (largest face flux x cells per unit xi).
* Fourth order (hc_level_prepare + hc_level_rhs, Berta WENOZ + Roe +
  Powell): the averaged metrics make the uniform state's residual a
  truncation error, not zero (the reference removes it for its magnetic
  test problems by subtracting the operator of the background).  Away from
  the radial boundaries (whose analytic-wind ghosts are not the uniform
  state) it must fall at least 2^4 from 16 to 32 cells per direction."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import make_box


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("riemann", [1, 2])
@pytest.mark.parametrize("vel", [0.0, 3.0e7])
def test_second_order_preserves_a_uniform_state(riemann, vel):
    _need_gpu()
    shell = hc.Shell(hc.Params(nr=12, na=10, limiter=3, riemann_solver=riemann))
    lo, hi, g, block = (3, 1, 2), (9, 8, 6), 2, 2
    v = [hi[d] - lo[d] + 1 for d in range(3)]
    w = np.zeros((8, v[2] + 2 * g, v[1] + 2 * g, v[0] + 2 * g))
    w[0], w[1], w[2], w[3], w[4] = 1e-20, vel, -0.5 * vel, 0.25 * vel, 1e-7
    w[5], w[6], w[7] = 1e-3, 2e-3, -1e-3
    nv = v[0] * v[1] * v[2]
    rhs = torch.zeros(8 * nv, dtype=torch.float64, device="cuda")
    fl = [torch.zeros(8 * (v[0] + (d == 0)) * (v[1] + (d == 1)) * (v[2] + (d == 2)), dtype=torch.float64,
                      device="cuda") for d in range(3)]
    shell.box_rhs(make_box(lo, hi, g, block), torch.from_numpy(w.reshape(-1).copy()).cuda(), rhs, fl, None, 1.0)
    torch.cuda.synchronize()
    r = rhs.cpu().numpy().reshape(8, -1)
    fmax = np.max([np.abs(f.cpu().numpy().reshape(8, -1)).max(axis=1) for f in fl], axis=0)
    scale = np.maximum(fmax * 12, 1e-300)   # face flux / cell width in xi (nr = 12 cells per unit xi0)
    assert np.isfinite(r).all()
    assert (np.abs(r).max(axis=1) <= 1e-12 * scale).all(), np.abs(r).max(axis=1) / scale


def _interior_residual(n):
    shell = hc.Shell(hc.Params(nr=n, na=n, spatial_order=4, riemann_solver=2, berta_fallback_type=0))
    det = shell.geometry(4).reshape(6, n, n)
    vol = shell.geometry(0).reshape(n + 1, 4)[:n, 3]
    J = det[:, :, :, None] * vol[None, None, None, :]
    U = np.array([1e-20, 0.0, 0.0, 0.0, 1e-7 / (5.0 / 3.0 - 1.0), 1e-3, 2e-3, -1e-3])
    U[4] += (1e-6 + 4e-6 + 1e-6) / (8 * np.pi)
    ju = torch.from_numpy(np.ascontiguousarray((J[:, None] * U[None, :, None, None, None]).reshape(-1))).cuda()
    k = shell.rhs(shell.prepare(ju, 0.0))
    torch.cuda.synchronize()
    kk = k.cpu().numpy().reshape(6, 8, n, n, n)[:, :, :, :, 6:n - 6]
    assert np.isfinite(kk).all()
    return np.abs(kk).reshape(6, 8, -1).max(axis=(0, 2))


def test_fourth_order_uniform_state_residual_converges():
    _need_gpu()
    r16, r32 = _interior_residual(16), _interior_residual(32)
    live = r16 > 0
    assert live.any()
    rates = np.log2(r16[live] / np.maximum(r32[live], 1e-300))
    assert (rates >= 4.0).all(), rates
