"""Served ensemble (heliocubed_b200.serve): every request's result is the
same alone (the plain per-solve path) and in the mix (the continuous-batching
server with pooled slots, CUDA-graph chunks and concurrent streams), admission
inserts the request's cone cloud on the device, and the server respects its
in-flight and HBM limits.

Tolerance: exact.  Both paths launch the same deterministic kernels on
buffers each request owns (the CFL max is order independent), so the final
states and model times agree bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    from heliocubed_b200 import serve


def _requests():
    return [
        serve.Request(0, 16, 16, 2, 12, 0.0, serve.Cone(1500, 40, 10, -20, 4)),
        serve.Request(1, 16, 16, 4, 12, 0.0, serve.Cone(800, 25, -15, 5, 3)),
        serve.Request(2, 20, 16, 2, 7, 0.0, serve.Cone(1200, 50, 0, 30, 5)),
        serve.Request(3, 16, 16, 4, 12, 0.01, serve.Cone(2000, 30, 20, 0, 2)),
        serve.Request(4, 16, 16, 2, 12, 0.02, serve.Cone(600, 20, -30, -30, 6)),
    ]


def _states(reqs, shells):
    out = {}
    for r in reqs:
        shp = (r.nr, r.na, r.order)
        if shp not in shells:
            shells[shp] = serve.Shell(r.params())
        out[r.rid] = serve.initial_state(shells[shp], r)
    return out


def test_results_same_alone_and_in_the_mix():
    if not gpu_available():
        pytest.skip("no CUDA device")
    reqs = _requests()
    shells = {}
    states = _states(reqs, shells)
    plain = {r.rid: r for r in serve.run_plain(reqs, shells=shells)}
    server = serve.EnsembleServer(hbm_budget=64e9, max_inflight=3, chunk=5)
    mixed = {r.rid: r for r in server.run(reqs)}
    assert set(plain) == set(mixed) == {r.rid for r in reqs}
    for rid in plain:
        a, b = plain[rid], mixed[rid]
        assert np.isfinite(a.state).all()
        assert a.model_time == b.model_time > 0
        assert np.array_equal(a.state, b.state), rid
        # the solve moved the admitted state (wind + inserted cloud)
        assert not np.array_equal(a.state, states[rid])


def test_admission_inserts_the_cloud():
    """Admission builds the wind and inserts the request's cloud: cells
    inside it carry the cloud's density; the rest is the wind."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    req = serve.Request(0, 16, 16, 4, 1, 0.0, serve.Cone(1500, 45, 10, 20, 4))
    sh = serve.Shell(req.params())
    ju = torch.from_numpy(serve.initial_state(sh, req)).cuda()
    wind = sh.init(serve.wind_spec())
    changed = (ju != wind).view(6, 8, -1).any(dim=1)
    assert int(changed.sum()) > 50
    cone = req.cone.prepared(sh.params)
    again = wind.clone()
    stats = sh.insert_cone(cone, cone.insertion_time, again, stats=True)
    assert int(stats[0].item()) == int(changed.sum())
    assert torch.equal(again, ju)


def test_budget_limits_inflight():
    if not gpu_available():
        pytest.skip("no CUDA device")
    reqs = [serve.Request(i, 16, 16, 2, 10, 0.0) for i in range(4)]
    server = serve.EnsembleServer(hbm_budget=64e9, max_inflight=4, chunk=5)
    server.warm(reqs, per_shape=1)
    one = server.slot_bytes[(16, 16, 2)]
    assert one > 0
    server.budget = 1.5 * one          # room for one solve at a time
    res = server.run(reqs)
    spans = sorted((r.t_start, r.t_done) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-3          # never two in flight
    assert len(server.pool[(16, 16, 2)]) == 1
