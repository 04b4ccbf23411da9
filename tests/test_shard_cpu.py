"""Radial slabs of one shell (heliocubed_b200.shard) on the host.

* The slab plan: owned ranges, halo layers, the columns each rank sends and
  receives, and the refusals.
* World sizes 2 and 3 over gloo: the sharded stepping code (ShardedShell with its
  point-to-point halo exchange and max all-reduce of the CFL rate) drives
  the oracle's level on each rank's slab; three RK4 steps with the shell's
  CFL dt equal the oracle's whole-shell steps bit for bit, at order 2
  (PLM-MC + Rusanov, Powell; 2 and 3 ranks, the middle one swapping with
  both neighbours) and order 4 (Berta WENOZ + Roe, Powell).  The
  reference exchanges ghost cells in each stage's preparation
  (src/BoxOp_SecondOrderPreStage.H:55) and reduces the CFL rate over ranks
  (src/BoxOp_SecondOrderCFL.H:207-209)."""
from __future__ import annotations

import os
import socket
import sys
import time

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)

from heliocubed_b200 import level as hl  # noqa: E402
from heliocubed_b200.shard import HALO, LocalTransport, ShardedShell, SlabPlan, slab_range  # noqa: E402

FIELDS = ("nr", "na", "spatial_order", "limiter", "riemann_solver", "divergence_cleaning", "sun_gravity", "cfl",
          "berta_fallback_type", "radial_offset", "radial_cells")
STEPS = 3
A4, B4 = (0.0, 0.5, 0.5, 1.0), (1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6)


def _params(order: int) -> hl.Params:
    if order == 2:
        return hl.Params(nr=16, na=8, spatial_order=2, limiter=3, riemann_solver=1, divergence_cleaning=1)
    return hl.Params(nr=24, na=16, spatial_order=4, riemann_solver=2, divergence_cleaning=1, berta_fallback_type=0)


class OracleSlab:
    """The oracle's level behind the per-stage interface ShardedShell drives
    (the order of operations of its own RK4 step)."""

    def __init__(self, p: hl.Params):
        from oracle import pyoracle as po
        self.p = p
        cp = po.make_params(**{f: getattr(p, f) for f in FIELDS})
        self.o = po.OracleLevelO4(cp) if p.spatial_order == 4 else po.OracleLevel(cp)
        self.n = 48 * p.na * p.na * p.nr
        self.stage = torch.zeros(self.n, dtype=torch.float64)

    def new_state(self) -> torch.Tensor:
        return torch.zeros(self.n, dtype=torch.float64)

    def stage_state(self, ju: torch.Tensor, s: int):
        return (ju if s == 0 else self.stage).view(-1, self.p.nr), 0

    def inv_dt_max(self, ju: torch.Tensor) -> torch.Tensor:
        return torch.tensor([self.o.inv_dt(ju.numpy())], dtype=torch.float64)

    def rk4_stage(self, ju, s, dt=0.0, t=0.0, inv_dt=None, time=None):
        if inv_dt is not None:
            dt = self.p.cfl / float(inv_dt[0])
        if time is not None:
            t = t + float(time[0])
        u = ju.numpy()
        src = u if s == 0 else self.stage.numpy()
        nxt = self.stage.numpy()
        if self.p.spatial_order == 2:
            if s == 0:
                self.k = []
            self.k.append(self.o.rhs(self.o.prepare(src, t + A4[s] * dt)))
            if s < 3:
                nxt[:] = u + (dt * A4[s + 1]) * self.k[s]
            else:
                for q in range(4):
                    u += (dt * B4[q]) * self.k[q]
            return
        if s == 0:
            self.acc, self.reg = u.copy(), self.o.register()
        k = self.o.rhs(self.o.prepare(src, t + A4[s] * dt), self.reg, dt * B4[s])
        self.acc += (dt * B4[s]) * k
        if s < 3:
            nxt[:] = u + (dt * A4[s + 1]) * k
        else:
            u[:] = self.acc
            self.o.reflux(self.reg, u)


def _whole_shell(order: int):
    """Initial state and the oracle's whole-shell steps: (ju0, [inv_dt], ju)."""
    from oracle import pyoracle as po
    p = _params(order)
    cp = po.make_params(**{f: getattr(p, f) for f in FIELDS})
    o = po.OracleLevelO4(cp) if order == 4 else po.OracleLevel(cp)
    base = o.base if order == 4 else o
    det = base.geometry(4).reshape(6, p.na, p.na)
    vol = base.geometry(0).reshape(p.nr + 1, 4)[:p.nr, 3]
    ju0 = np.ascontiguousarray(hl.perturbed_wind_state(p, det, vol, seed=77).reshape(-1))
    ju, invs = ju0.copy(), []
    for _ in range(STEPS):
        invs.append(o.inv_dt(ju))
        o.rk4_step(ju, p.cfl / invs[-1], 0.0)
    return ju0, invs, ju


def test_slab_plan():
    assert [slab_range(26, 3, r) for r in range(3)] == [(0, 8), (8, 17), (17, 26)]
    p0, p1, p2 = (SlabPlan(26, 3, r, 2) for r in range(3))
    assert (p0.below, p0.above, p0.local_nr, p0.offset) == (0, 2, 10, 0)
    assert (p1.below, p1.above, p1.local_nr, p1.offset) == (2, 2, 13, 6)
    assert (p2.below, p2.above, p2.local_nr, p2.offset) == (2, 0, 11, 15)
    # rank 1 (first level cell at column 3): sends its first and last 2 owned
    # columns, receives 2 halo columns on each side
    assert p1.links(3) == [(0, slice(5, 7), slice(3, 5)), (2, slice(12, 14), slice(14, 16))]
    assert p0.links(0) == [(1, slice(6, 8), slice(8, 10))]
    assert p2.links(0) == [(1, slice(2, 4), slice(0, 2))]
    sp = p1.params(hl.Params(nr=26, na=8))
    assert (sp.nr, sp.radial_offset, sp.radial_cells) == (13, 6, 26)
    assert HALO == {2: 2, 4: 6}
    with pytest.raises(ValueError):
        SlabPlan(20, 4, 0, 6)                      # 5 owned cells < halo 6
    with pytest.raises(ValueError):
        SlabPlan(20, 2, 2, 2)                      # no such rank
    with pytest.raises(ValueError):
        p1.params(sp)                              # a slab is not split again
    with pytest.raises(ValueError):                # two of three slabs in one process
        ShardedShell(hl.Params(nr=24, na=8), 0, 3, level=lambda p: None, ranks=[0, 1])
    with pytest.raises(ValueError):                # a slab twice
        ShardedShell(hl.Params(nr=24, na=8), 0, 2, level=lambda p: None, ranks=[0, 0])


def test_local_exchange_moves_owned_layers_into_halos():
    """Three host slabs, halo 2: every halo column ends up holding its
    neighbour's owned column of the same radial cell, owned columns stay."""
    nr, world, h, rows = 15, 3, 2, 4
    plans = [SlabPlan(nr, world, r, h) for r in range(world)]
    bufs = []
    for p in plans:
        b = torch.full((rows, p.local_nr + 4), -1.0, dtype=torch.float64)   # 2 ghost columns each side
        for c in range(p.below, p.below + p.hi - p.lo):
            b[:, 2 + c] = p.offset + c + 1000 * torch.arange(rows)
        bufs.append((b, 2))
    LocalTransport().exchange(plans, bufs)
    for p, (b, first) in zip(plans, bufs):
        for c in range(p.local_nr):
            assert torch.equal(b[:, first + c], p.offset + c + 1000 * torch.arange(rows, dtype=torch.float64))
        assert (b[:, :first] == -1).all() and (b[:, first + p.local_nr:] == -1).all()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, order, ju0, q, advance=False):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _params(order)
        sh = ShardedShell(p, rank, world, level=OracleSlab)
        states = sh.scatter(torch.from_numpy(ju0))
        invs = []
        if advance:
            # dt kept as a tensor: the all-reduce feeds the stages directly
            time = torch.zeros(1, dtype=torch.float64)
            sh.advance(states, STEPS, time)
            invs = [float(time[0])]
        else:
            for _ in range(STEPS):
                inv = sh.inv_dt_max(states)
                invs.append(float(inv[0]))
                sh.rk4_step(states, p.cfl / invs[-1], 0.0)
        q.put((rank, sh.plans[0].lo, sh.owned(states)[0].numpy().copy(), invs))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("order,world,advance", [(2, 2, False), (2, 3, False), (2, 2, True), (4, 2, False)])
def test_rank_slabs_step_like_the_whole_shell(order, world, advance, oracle_lib):
    ju0, invs_want, want = _whole_shell(order)
    if advance:
        t = 0.0
        for inv in invs_want:
            t += _params(order).cfl / inv
        invs_want = [t]
    p = _params(order)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, order, ju0, q, advance)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = sorted((q.get(timeout=600) for _ in range(world)), key=lambda x: x[0])
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    want = want.reshape(6, 8, p.na, p.na, p.nr)
    for rank, lo, owned, invs in got:
        assert invs == invs_want, (rank, invs, invs_want)
        assert np.array_equal(owned, want[..., lo:lo + owned.shape[-1]]), rank
    assert sum(x[2].shape[-1] for x in got) == p.nr


def _mismatch_worker(rank, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        p = _params(2)
        if rank == 1:
            p = hl.Params(**{**vars(p), "cfl": 0.3})        # one rank with another CFL number
        try:
            ShardedShell(p, rank, 2, level=OracleSlab)
            q.put((rank, "built"))
        except ValueError as e:
            q.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


def test_ranks_with_different_shells_refuse_to_start(oracle_lib):
    """Every rank raises before any halo swap when one rank's parameters
    differ (its buffers would not match its neighbours')."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mismatch_worker, args=(r, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert [r for r, _ in got] == [0, 1]
    assert all("split a different shell" in msg for _, msg in got), got


def _resume_worker(rank, port, ju0, path, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        p = _params(2)
        sh = ShardedShell(p, rank, 2, level=OracleSlab)
        states = sh.scatter(torch.from_numpy(ju0))
        for _ in range(STEPS - 1):
            sh.rk4_step(states, p.cfl / float(sh.inv_dt_max(states)[0]), 0.0)
        sh.save(path, states, time=1.5, step=STEPS - 1, attributes={"cme_inserted_count": 0})
        fresh = ShardedShell(p, rank, 2, level=OracleSlab)           # a restarted job
        states, time, step, attrs = fresh.load(path)
        fresh.rk4_step(states, p.cfl / float(fresh.inv_dt_max(states)[0]), 0.0)
        q.put((rank, fresh.plans[0].lo, fresh.owned(states)[0].numpy().copy(), (time, step, attrs)))
    finally:
        dist.destroy_process_group()


def test_sharded_checkpoint_resumes_exactly(oracle_lib, tmp_path):
    """Two ranks step, write one whole-shell checkpoint (rank 0 collects the
    owned cells), restart from it and step again: the same cells as the
    oracle's uninterrupted whole-shell run, bit for bit, and the file is
    the whole shell's state after the first steps."""
    from heliocubed_b200 import checkpoint
    ju0, invs, want = _whole_shell(2)
    p = _params(2)
    path = str(tmp_path / "slabs.ck")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_resume_worker, args=(r, port, ju0, path, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = sorted((q.get(timeout=300) for _ in range(2)), key=lambda x: x[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    want = want.reshape(6, 8, p.na, p.na, p.nr)
    for rank, lo, owned, meta in got:
        assert meta == (1.5, STEPS - 1, {"cme_inserted_count": 0})
        assert np.array_equal(owned, want[..., lo:lo + owned.shape[-1]]), rank
    from oracle import pyoracle as po
    o = po.OracleLevel(po.make_params(**{f: getattr(p, f) for f in FIELDS}))
    mid = ju0.copy()
    for inv in invs[:STEPS - 1]:
        o.rk4_step(mid, p.cfl / inv, 0.0)
    params, state, _, _, _ = checkpoint.load(path)
    assert params == p and np.array_equal(state, mid)


def test_emulated_slabs_checkpoint_round_trip(oracle_lib, tmp_path):
    """A checkpoint written by three slabs in one process is the whole
    shell's state; two slabs load it back with their halo layers; another
    shell's checkpoint is refused."""
    from heliocubed_b200 import checkpoint
    ju0, _, _ = _whole_shell(2)
    p = _params(2)
    path = str(tmp_path / "three.ck")
    three = ShardedShell.emulated(p, 3, level=OracleSlab)
    three.save(path, three.scatter(torch.from_numpy(ju0)), time=2.0, step=7)
    _, state, time, step, _ = checkpoint.load(path)
    assert np.array_equal(state, ju0) and (time, step) == (2.0, 7)
    two = ShardedShell.emulated(p, 2, level=OracleSlab)
    states, _, _, _ = two.load(path)
    full = ju0.reshape(6, 8, p.na, p.na, p.nr)
    for plan, st in zip(two.plans, states):
        assert np.array_equal(st.numpy().reshape(6, 8, p.na, p.na, plan.local_nr),
                              full[..., plan.offset:plan.offset + plan.local_nr])
    other = ShardedShell.emulated(hl.Params(**{**vars(p), "cfl": 0.3}), 2, level=OracleSlab)
    with pytest.raises(checkpoint.CheckpointError):
        other.load(path)


def _leaving_worker(rank, port, ju0, q):
    import datetime
    import torch.distributed as dist
    from heliocubed_b200.shard import SlabExchangeError
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=10))
    p = _params(2)
    sh = ShardedShell(p, rank, 2, level=OracleSlab)
    states = sh.scatter(torch.from_numpy(ju0))
    sh.rk4_step(states, 1.0e3, 0.0)
    def report(msg):
        q.put((rank, msg))
        q.close()
        q.join_thread()                               # flushed before the hard exit below

    if rank == 1:
        report("left")
        os._exit(0)                                   # leaves between steps, with nothing in flight
    t0 = time.monotonic()
    try:
        sh.rk4_step(states, 1.0e3, 0.0)
        report("stepped")
    except SlabExchangeError as e:
        report(f"error after {time.monotonic() - t0:.1f} s: {e}")
    os._exit(0)


def test_a_rank_that_leaves_fails_the_next_swap(oracle_lib):
    """Failure detection on the host: rank 1 exits between steps; rank 0's
    next halo swap raises SlabExchangeError within the process group's
    timeout instead of waiting for ever."""
    ju0, _, _ = _whole_shell(2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, port, ju0, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for pr in procs:
        pr.join(timeout=60)
    assert got[1] == "left"
    assert got[0].startswith("error after") and "halo swap with ranks [1]" in got[0], got[0]
    assert float(got[0].split()[2]) < 30.0
