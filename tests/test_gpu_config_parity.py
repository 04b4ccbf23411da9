"""Parity at the workloads' own sizes and step counts: the CUDA path through
the C ABI against the oracle, each advancing with its own CFL time step
(the device takes dt = cfl / max rate on the GPU every step, the oracle on
the host), as the reference driver's step loop does (exec/main.cpp:369-497).

* second order, the full 32 x 32^2 x 6 shell with PLM-MC + Rusanov and the
  seeded pressure pulse, 10 RK4 steps at CFL 0.4: <= 1e-10 per component;
* fourth order (Berta pointwise WENOZ + Roe 8-wave + Powell), 32 x 32^2 x 6
  on the perturbed Parker-like wind, 5 RK4 steps: <= 1e-10 per component;
* fourth order at 16 x 16^2 x 6 for 100 RK4 steps: <= 1e-10 per component.

Each also checks the conserved totals (sum of mass, momentum, energy and
field over the shell) against the oracle's to round-off of the summed
magnitudes, and the accumulated time.  Tolerances are normwise per
component, max|gpu - oracle| / max|oracle|; the device contracts a*b+c
into FMA where the oracle does not, so the two agree to accumulated
round-off rather than bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200 import level as hl

SEED = 20261204


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _totals_close(got: np.ndarray, ref: np.ndarray, tol: float = 1e-12) -> np.ndarray:
    g = got.reshape(6, 8, -1)
    r = ref.reshape(6, 8, -1)
    diff = np.abs(g.sum(axis=(0, 2)) - r.sum(axis=(0, 2)))
    mag = np.abs(r).sum(axis=(0, 2))
    return diff <= tol * np.maximum(mag, 1e-300)


def _advance_both(shell, orc, ju: np.ndarray, nsteps: int, cfl: float = 0.4):
    g = torch.from_numpy(ju.copy()).cuda()
    time = torch.zeros(1, dtype=torch.float64, device="cuda")
    shell.advance(g, nsteps, time)
    t = 0.0
    for _ in range(nsteps):
        dt = cfl / orc.inv_dt(ju)
        orc.rk4_step(ju, dt, t)
        t += dt
    torch.cuda.synchronize()
    return g, float(time.item()), t


def test_config1_full_shell_ten_steps(oracle_lib):
    """PLM-MC + Rusanov on the whole 32 x 32^2 x 6 shell, 10 RK4 steps."""
    _need_gpu()
    nr = na = 32
    kw = dict(nr=nr, na=na, limiter=3, riemann_solver=1, divergence_cleaning=1, sun_gravity=0, cfl=0.4)
    shell = hc.Shell(hc.Params(**kw))
    orc = oracle_lib.OracleLevel(oracle_lib.make_params(**kw))
    spec = hc.InitSpec.seeded(SEED, nr, na)
    init = oracle_lib.HcInit()
    init.kind = 1
    for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref", "pulse_amp",
              "pulse_width"):
        setattr(init, k, getattr(spec, k))
    ju = orc.init(init)
    g, t_gpu, t_orc = _advance_both(shell, orc, ju, 10)
    got = g.cpu().numpy()
    err = rel_err_components(got.reshape(6, 8, -1), ju.reshape(6, 8, -1))
    assert np.isfinite(got).all() and shell.valid(g) and orc.valid(ju)
    assert abs(t_gpu - t_orc) <= 1e-12 * t_orc
    assert err.max() <= 1e-10, err
    assert _totals_close(got, ju).all()
    shell.close()


def _o4_pair(oracle_lib, n: int):
    kw = dict(nr=n, na=n, spatial_order=4, riemann_solver=2, divergence_cleaning=1, sun_gravity=0,
              berta_fallback_type=0, cfl=0.4)
    shell = hc.Shell(hc.Params(**kw))
    orc = oracle_lib.OracleLevelO4(oracle_lib.make_params(**kw))
    det = orc.base.geometry(4).reshape(6, n, n)
    vol = orc.base.geometry(0).reshape(n + 1, 4)[:n, 3]
    ju = np.ascontiguousarray(hl.perturbed_wind_state(hl.Params(**kw), det, vol, seed=SEED).reshape(-1))
    return shell, orc, ju


@pytest.mark.parametrize("n,nsteps", [(32, 5), (16, 100)])
def test_o4_wenoz_roe_multistep(oracle_lib, n, nsteps):
    """Berta WENOZ + Roe 8-wave + Powell: 5 steps at 32^3 x 6, 100 at 16^3 x 6."""
    _need_gpu()
    shell, orc, ju = _o4_pair(oracle_lib, n)
    g, t_gpu, t_orc = _advance_both(shell, orc, ju, nsteps)
    got = g.cpu().numpy()
    err = rel_err_components(got.reshape(6, 8, -1), ju.reshape(6, 8, -1))
    assert np.isfinite(got).all() and shell.valid(g)
    assert abs(t_gpu - t_orc) <= 1e-11 * t_orc
    assert err.max() <= 1e-10, err
    assert _totals_close(got, ju).all()
    shell.close()
