"""Autotuner on the GPU (hc_ctx_autotune, hc_ctx_set_tiles,
hc_ctx_set_o4_variants).  Order 2: every candidate tile of the stage kernel
gives bit-identical RK4 steps and operator results (the tile only changes
which CTA computes a face), the tuner leaves the state untouched and picks a
timed candidate, and automatic tuning on the first step changes no result
(exact).  Order 4: the register-cap variants agree to round-off (1e-13)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import stage_tiles


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


SCHEMES = [dict(limiter=3, riemann_solver=1), dict(limiter=1, riemann_solver=2),
           dict(limiter=3, riemann_solver=2, sun_gravity=1)]


@pytest.mark.parametrize("scheme", SCHEMES)
def test_every_tile_gives_identical_results(scheme):
    _need_gpu()
    sh = hc.Shell(hc.Params(nr=20, na=12, **scheme))
    ju0 = sh.init(hc.InitSpec.seeded(3, 20, 12))
    ref_state = ref_rhs = None
    for t in range(stage_tiles().shape[0]):
        sh.set_tiles(t, t)
        ju = ju0.clone()
        time = torch.zeros(1, dtype=torch.float64, device="cuda")
        sh.advance(ju, 2, time)
        k = sh.rhs(sh.prepare(ju0))
        torch.cuda.synchronize()
        if ref_state is None:
            ref_state, ref_rhs = ju, k
        else:
            assert torch.equal(ju, ref_state), t
            assert torch.equal(k, ref_rhs), t


def test_autotune_picks_a_timed_tile_and_keeps_the_state():
    _need_gpu()
    sh = hc.Shell(hc.Params(nr=32, na=32))
    ju = sh.init(hc.InitSpec.seeded(1, 32, 32))
    before = ju.clone()
    (trk, trhs), ms = sh.autotune(ju)
    n = stage_tiles().shape[0]
    assert 0 <= trk < n and 0 <= trhs < n
    assert ms.shape == (2, n) and (ms > 0).all()
    assert ms[0, trk] == ms[0].min() and ms[1, trhs] == ms[1].min()
    assert torch.equal(ju, before)


def test_automatic_tuning_changes_no_result():
    _need_gpu()
    plain = hc.Shell(hc.Params(nr=24, na=16))
    tuned = hc.Shell(hc.Params(nr=24, na=16, autotune=1))
    ju0 = plain.init(hc.InitSpec.seeded(2, 24, 16))
    a, b = ju0.clone(), ju0.clone()
    ta = torch.zeros(1, dtype=torch.float64, device="cuda")
    tb = torch.zeros(1, dtype=torch.float64, device="cuda")
    plain.advance(a, 3, ta)
    tuned.advance(b, 3, tb)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(ta, tb)


def test_o4_variants_agree_and_tune():
    """Every register-cap variant of the fourth-order operator's tuned
    kernels gives the same level step to round-off (1e-13 normwise per
    component: the code generator contracts multiply-adds per variant), and
    the tuner picks the fastest timed variant of each without touching the
    state; with the variant fixed, steps repeat bit for bit."""
    _need_gpu()
    from conftest import rel_err_components
    sh = hc.Shell(hc.Params(nr=16, na=16, spatial_order=4, riemann_solver=2))
    ju0 = sh.init_perturbed_wind(4)
    ref = None
    for v in range(3):
        sh.set_o4_variants(v, v, v)
        ju = ju0.clone()
        sh.rk4_step(ju, 50.0, 0.0)
        again = ju0.clone()
        sh.rk4_step(again, 50.0, 0.0)
        torch.cuda.synchronize()
        assert torch.equal(ju, again), v
        if ref is None:
            ref = ju
        else:
            err = rel_err_components(ju.cpu().numpy().reshape(6, 8, -1), ref.cpu().numpy().reshape(6, 8, -1))
            assert err.max() < 1e-13, (v, err)
    before = ju0.clone()
    var, ms = sh.autotune(ju0)
    assert torch.equal(ju0, before)
    assert ms.shape == (3, 3) and (ms > 0).all()
    for q in range(3):
        assert ms[q, var[q]] == ms[q].min()
