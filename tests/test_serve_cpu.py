"""Host logic of the served ensemble (heliocubed_b200.serve.EnsembleServer)
on the CPU: admission under the HBM budget and the in-flight cap,
continuous batching (a request that arrives while others run starts before
they finish), slot pooling by shape, and the result bookkeeping.

The device work of a slot is simulated: `FakeSlot` has the interface of
`serve.Slot` (start, issue, an event to poll, the host result buffers) and
completes each issued chunk after a fixed wall time, so the scheduler runs
exactly as it does over CUDA streams."""
import threading
import time
import types

import numpy as np
import pytest

from heliocubed_b200 import serve

CHUNK_S = 0.004  # wall time of one simulated chunk


class FakeEvent:
    def __init__(self, ready: float):
        self.ready = ready

    def query(self) -> bool:
        return time.perf_counter() >= self.ready


class FakeSlot:
    built = 0
    active = 0
    max_active = 0
    lock = threading.Lock()
    bytes_per_cell = 64.0

    def __init__(self, shape, chunk, device, graph=True):
        nr, na, _ = shape
        self.shape = shape
        self.chunk = chunk
        self.bytes = int(6 * nr * na * na * self.bytes_per_cell)
        self.req = None
        self.left = 0
        self.event = None
        self.t_start = 0.0
        self.host_out = None
        self.host_time = None
        self.in_cohort = False
        self.stream = None
        self.graph = None
        self.shell = types.SimpleNamespace(close=lambda: None)
        FakeSlot.built += 1

    def start(self, req, now):
        self.req = req
        self.left = req.steps
        self.t_start = now
        self.event = None
        with FakeSlot.lock:
            FakeSlot.active += 1
            FakeSlot.max_active = max(FakeSlot.max_active, FakeSlot.active)

    def issue(self):
        if self.left >= self.chunk:
            self.left -= self.chunk
        elif self.left > 0:
            self.left = 0
        else:
            # the result copy: a state that records which request it was
            self.host_out = _Host(np.full(4, float(self.req.rid)))
            self.host_time = _Host(np.array(float(self.req.steps)))
            self.left = -1
            with FakeSlot.lock:
                FakeSlot.active -= 1
        self.event = FakeEvent(time.perf_counter() + CHUNK_S)


class _Host:
    def __init__(self, a):
        self.a = a

    def numpy(self):
        return self.a

    def item(self):
        return float(self.a)


@pytest.fixture
def fake_slots(monkeypatch):
    FakeSlot.built = FakeSlot.active = FakeSlot.max_active = 0
    monkeypatch.setattr(serve, "Slot", FakeSlot)
    return FakeSlot


def _req(rid, nr=8, na=8, steps=30, arrival=0.0):
    return serve.Request(rid, nr, na, 2, steps, arrival)


def _slot_bytes(nr=8, na=8):
    return 6 * nr * na * na * FakeSlot.bytes_per_cell


def test_budget_limits_admitted_solves(fake_slots):
    reqs = [_req(i) for i in range(6)]
    srv = serve.EnsembleServer(hbm_budget=2.5 * _slot_bytes(), max_inflight=8, chunk=10, device=0)
    srv.warm(reqs)
    res = srv.run(reqs)
    assert sorted(r.rid for r in res) == list(range(6))
    assert fake_slots.max_active == 2          # two slots fit the budget
    assert srv.in_use == 0                     # every slot released
    for r in res:
        assert r.state[0] == r.rid and r.model_time == r.steps


def test_inflight_cap(fake_slots):
    reqs = [_req(i) for i in range(7)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=3, chunk=10, device=0)
    srv.warm(reqs)
    res = srv.run(reqs)
    assert len(res) == 7 and fake_slots.max_active == 3


def test_late_arrival_joins_while_others_run(fake_slots):
    # one long solve from t = 0, a short one arriving at 20 ms: it is admitted
    # at once and finishes while the long one is still running
    long_req = _req(0, steps=400)              # 40 chunks of 4 ms
    short_req = _req(1, steps=20, arrival=0.02)
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=4, chunk=10, device=0)
    srv.warm([long_req, short_req], per_shape=2)
    res = {r.rid: r for r in srv.run([long_req, short_req])}
    assert res[1].t_start >= 0.02
    # not queued behind the long solve (160 ms of chunks)
    assert res[1].t_start < res[0].t_done - 0.05
    assert res[1].t_done < res[0].t_done
    assert fake_slots.max_active == 2


def test_slots_pooled_by_shape(fake_slots):
    reqs = [_req(i, arrival=0.03 * i) for i in range(4)] + [_req(10, nr=16, na=8, arrival=0.0)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=8, chunk=10, device=0)
    srv.warm(reqs)
    built = fake_slots.built
    assert built == 2                          # one slot per shape
    res = srv.run(reqs)
    assert len(res) == 5
    # the spaced same-shape requests reuse pooled slots (each normally
    # finishes before the next arrives): far fewer builds than requests
    assert fake_slots.built - built <= 2


def test_summary_of_results(fake_slots):
    reqs = [_req(i, steps=20) for i in range(5)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=5, chunk=10, device=0)
    srv.warm(reqs)
    s = serve.summarize(srv.run(reqs))
    assert s["requests"] == 5 and s["cell_updates"] == 5 * 20 * 6 * 8 * 8 * 8
    assert 0 < s["p50_s"] <= s["p99_s"] <= s["makespan_s"] + 1e-9


def test_request_over_the_budget_is_refused(fake_slots):
    """A request whose slot alone needs more than the budget is refused with
    an error naming the sizes; the others are served and the loop ends."""
    small = [_req(i) for i in range(3)]
    big = _req(9, nr=32, na=32)
    srv = serve.EnsembleServer(hbm_budget=2.5 * _slot_bytes(), max_inflight=8, chunk=10, device=0)
    srv.warm(small + [big])
    res = {r.rid: r for r in srv.run(small + [big])}
    assert sorted(res) == [0, 1, 2, 9]
    assert res[9].error is not None and "budget" in res[9].error and res[9].state.size == 0
    assert all(res[i].error is None and res[i].state[0] == i for i in range(3))
    assert serve.summarize(list(res.values()))["requests"] == 3
    assert srv.in_use == 0


def test_unseen_shape_admitted_by_estimate(fake_slots):
    """A shape with no built slot is admitted by an estimate scaled from the
    measured slots of its order, not with a size of zero."""
    srv = serve.EnsembleServer(hbm_budget=3.5 * _slot_bytes(), max_inflight=8, chunk=10, device=0)
    srv.warm([_req(0)])
    assert srv.estimate_bytes((16, 8, 2)) == 2 * _slot_bytes()
    reqs = [_req(0, steps=200), _req(1, steps=200), _req(2, nr=16, steps=20)]
    res = {r.rid: r for r in srv.run(reqs)}
    # the two small solves hold 2 of 3.5 budget units; the unseen 2-unit shape
    # waits for one of them instead of being built past the budget
    assert res[2].t_start >= min(res[0].t_done, res[1].t_done) - 1e-3
    assert all(r.error is None for r in res.values())


class FakeEnsemble:
    def __init__(self, rids):
        self.rids = rids
        self.closed = False

    def close(self):
        self.closed = True


class FakeCohort(serve.Cohort):
    """serve.Cohort with its device calls simulated: a chunk completes
    CHUNK_S after its launch, admissions at once."""
    launches = []
    built = []

    def _new_stream(self):
        return "cohort"

    @staticmethod
    def _record(stream):
        return FakeEvent(time.perf_counter() + (CHUNK_S if stream == "cohort" else 0.0))

    @staticmethod
    def _wait(stream, event):
        assert event.query()  # the scheduler waits only on completed work

    @staticmethod
    def _ensemble(slots):
        ens = FakeEnsemble(tuple(s.req.rid for s in slots))
        FakeCohort.built.append(ens)
        return ens

    def _advance(self, ens, slots, steps):
        FakeCohort.launches.append(([s.req.rid for s in slots], steps, [s.left for s in slots]))


def test_fourth_order_requests_step_as_one_cohort(fake_slots, monkeypatch):
    """Fourth-order requests of different sizes step together in chunks of
    min(chunk, fewest steps left); one that finishes leaves with its result,
    a late arrival joins at a chunk boundary; second-order requests keep
    their own slots; every request gets exactly its steps."""
    FakeCohort.launches, FakeCohort.built = [], []
    monkeypatch.setattr(serve, "Cohort", FakeCohort)
    reqs = [serve.Request(0, 8, 8, 4, 45, 0.0), serve.Request(1, 16, 8, 4, 15, 0.0),
            serve.Request(2, 8, 8, 2, 20, 0.0), serve.Request(3, 8, 8, 4, 10, 0.006)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=8, chunk=10, device=0)
    srv.warm(reqs, per_shape=2)
    res = {r.rid: r for r in srv.run(reqs)}
    assert sorted(res) == [0, 1, 2, 3]
    assert all(r.state[0] == r.rid and r.model_time == r.steps for r in res.values())
    stepped = {0: 0, 1: 0, 3: 0}
    for rids, steps, left in FakeCohort.launches:
        assert 2 not in rids                       # second order never joins
        assert steps == min(10, min(left))         # lockstep chunk
        for rid in rids:
            stepped[rid] += steps
    assert stepped == {0: 45, 1: 15, 3: 10}
    assert FakeCohort.launches[0][0] == [0, 1]     # both arrivals at t = 0 start together
    assert any(3 in rids and 0 in rids for rids, _, _ in FakeCohort.launches)  # the late one joined
    assert len(FakeCohort.built) == len({tuple(r) for r, _, _ in FakeCohort.launches})
    srv.close()
    assert all(e.closed for e in FakeCohort.built)
    assert srv.in_use == 0


def test_cobatch_off_keeps_per_slot_chunks(fake_slots, monkeypatch):
    FakeCohort.launches = []
    monkeypatch.setattr(serve, "Cohort", FakeCohort)
    reqs = [serve.Request(0, 8, 8, 4, 20, 0.0), serve.Request(1, 8, 8, 4, 20, 0.0)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=8, chunk=10, device=0, cobatch=False)
    srv.warm(reqs, per_shape=2)
    res = srv.run(reqs)
    assert len(res) == 2 and FakeCohort.launches == []


def test_cohort_keeps_a_bounded_number_of_ensembles(fake_slots, monkeypatch):
    """Past max_kept memberships the least recently used ensemble is
    released (between chunks, never the running one)."""
    FakeCohort.launches, FakeCohort.built = [], []
    monkeypatch.setattr(serve, "Cohort", FakeCohort)
    monkeypatch.setattr(FakeCohort, "max_kept", 2)
    reqs = [serve.Request(i, 8, 8, 4, 10 + 5 * (i % 3), 0.003 * i) for i in range(8)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=3, chunk=5, device=0)
    srv.warm(reqs, per_shape=4)
    res = srv.run(reqs)
    assert len(res) == 8 and all(r.state[0] == r.rid for r in res)
    assert len(FakeCohort.built) > 2                  # memberships changed past the bound
    assert len(srv.cohort.ensembles) <= 2
    closed = [e for e in FakeCohort.built if e.closed]
    assert len(closed) == len(FakeCohort.built) - len(srv.cohort.ensembles)
    srv.close()


def test_forget_ensembles_rebuilds_memberships(fake_slots, monkeypatch):
    """A second run of the same stream finds every membership cached unless
    the cohort's ensembles are released between the runs; after release it
    builds them again, as the first run did."""
    FakeCohort.launches, FakeCohort.built = [], []
    monkeypatch.setattr(serve, "Cohort", FakeCohort)
    reqs = [serve.Request(i, 8, 8, 4, 10, 0.002 * i) for i in range(4)]
    srv = serve.EnsembleServer(hbm_budget=1e18, max_inflight=4, chunk=5, device=0)
    srv.warm(reqs, per_shape=4)
    srv.run(reqs)
    first = len(FakeCohort.built)
    srv.run(reqs)
    cached = len(FakeCohort.built) - first
    srv.forget_ensembles()
    assert srv.cohort.ensembles == {} and all(e.closed for e in FakeCohort.built)
    before = len(FakeCohort.built)
    srv.run(reqs)
    assert first > 0 and len(FakeCohort.built) - before > 0 and cached <= len(FakeCohort.built) - before
    srv.close()
