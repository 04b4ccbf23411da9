"""Ensemble stepping (hc_ensemble): fourth-order levels of different sizes,
each with its own cone cloud and insertion schedule (CFL ramp and Rusanov
window), advanced together with every stage operator batched over all their
panels, against each level advanced alone (hc_level_advance_cfl).

Tolerance: exact.  The batched operator runs the same per-box arithmetic on
the same buffers (its tiling and work lists change, not the order of any
sum), so states, model times and dts agree bit for bit.
"""
from __future__ import annotations

import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200._native as N
    from heliocubed_b200 import level as hl
    from heliocubed_b200 import serve


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


REQS = [
    (16, 16, (1500, 40, 10, -20, 4)),
    (24, 16, (800, 25, -15, 5, 3)),
    (16, 20, (2000, 30, 20, 0, 2)),
]


def _admitted(nr, na, cone):
    req = serve.Request(0, nr, na, 4, 0, 0.0, serve.Cone(*cone))
    sh = hl.Shell(req.params())
    ju = sh.new_state()
    t = torch.zeros(1, dtype=torch.float64, device=ju.device)
    serve.admit(sh, req, ju, t)
    return sh, ju, t


def test_ensemble_equals_levels_alone():
    _need_gpu()
    alone, together = [], []
    for nr, na, cone in REQS:
        alone.append(_admitted(nr, na, cone))
        together.append(_admitted(nr, na, cone))
    for (_, a, _), (_, b, _) in zip(alone, together):
        assert torch.equal(a, b)
    dts_a = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in REQS]
    dts_b = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in REQS]
    for (sh, ju, t), dt in zip(alone, dts_a):
        sh.advance(ju, 3, t, dt)
        sh.advance(ju, 4, t, dt)
    ens = hl.Ensemble([sh for sh, _, _ in together])
    ens.advance([ju for _, ju, _ in together], 3, [t for _, _, t in together], dts_b)
    ens.advance([ju for _, ju, _ in together], 4, [t for _, _, t in together], dts_b)
    torch.cuda.synchronize()
    for q, ((sha, a, ta), (_, b, tb)) in enumerate(zip(alone, together)):
        assert torch.isfinite(a).all() and sha.valid(a)
        assert float(ta.item()) > 0
        assert torch.equal(ta, tb), q
        assert torch.equal(dts_a[q], dts_b[q]), q
        assert torch.equal(a, b), (q, (a - b).abs().max().item())
    ens.close()


def test_ensemble_graph_replay_matches_eager():
    """A captured ensemble chunk replays the eager launch sequence."""
    _need_gpu()
    eager = [_admitted(nr, na, cone) for nr, na, cone in REQS[:2]]
    graph = [_admitted(nr, na, cone) for nr, na, cone in REQS[:2]]
    e1 = hl.Ensemble([sh for sh, _, _ in eager])
    e2 = hl.Ensemble([sh for sh, _, _ in graph])
    e1.advance([ju for _, ju, _ in eager], 4, [t for _, _, t in eager])
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    states, times = [ju for _, ju, _ in graph], [t for _, _, t in graph]
    saved = [s.clone() for s in states], [t.clone() for t in times]
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        e2.advance(states, 2, times)  # warm-up off the capture
    torch.cuda.current_stream().wait_stream(side)
    for s, s0 in zip(states, saved[0]):
        s.copy_(s0)
    for t, t0 in zip(times, saved[1]):
        t.copy_(t0)
    with torch.cuda.graph(g):
        e2.advance(states, 2, times)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for (_, a, ta), (_, b, tb) in zip(eager, graph):
        assert torch.equal(ta, tb)
        assert torch.equal(a, b)
    g = None
    e1.close()
    e2.close()


def test_ensemble_refuses_mixed_schemes_and_repeats():
    _need_gpu()
    o4 = hl.Shell(hl.Params(nr=16, na=16, spatial_order=4, riemann_solver=2, berta_fallback_type=0))
    o2 = hl.Shell(hl.Params(nr=12, na=12))
    rus = hl.Shell(hl.Params(nr=16, na=16, spatial_order=4, riemann_solver=1, berta_fallback_type=0))
    for members in ([o4, o2], [o4, o4], [o4, rus]):
        with pytest.raises(N.HcError):
            hl.Ensemble(members)


@pytest.mark.parametrize("riemann,gravity", [(2, 1), (1, 0)])
def test_ensemble_other_schemes_equal_levels_alone(riemann, gravity):
    """Gravity (batched over the ensemble's panels) and the Rusanov solver:
    the ensemble equals each level alone, bit for bit."""
    _need_gpu()
    kw = dict(spatial_order=4, riemann_solver=riemann, sun_gravity=gravity, berta_fallback_type=0)
    sizes = [(16, 16), (20, 16)]
    alone, together = [], []
    for q, (nr, na) in enumerate(sizes):
        for group in (alone, together):
            sh = hl.Shell(hl.Params(nr=nr, na=na, **kw))
            ju = sh.init_perturbed_wind(7 + q)
            t = torch.zeros(1, dtype=torch.float64, device=ju.device)
            group.append((sh, ju, t))
    for sh, ju, t in alone:
        sh.advance(ju, 3, t)
    ens = hl.Ensemble([sh for sh, _, _ in together])
    ens.advance([ju for _, ju, _ in together], 3, [t for _, _, t in together])
    torch.cuda.synchronize()
    for (sha, a, ta), (_, b, tb) in zip(alone, together):
        assert torch.isfinite(a).all() and sha.valid(a)
        assert torch.equal(ta, tb)
        assert torch.equal(a, b)
    ens.close()
