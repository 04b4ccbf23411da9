"""One shell split into radial slabs, one per rank (one process per GPU).

The reference spreads each panel's boxes over MPI ranks (Proto's
DisjointBoxLayout), exchanges the ghost cells of the stage primitives between
boxes and ranks in every stage's preparation
(src/BoxOp_SecondOrderPreStage.H:55) and takes dt from the maximum over ranks
of the CFL rate (src/BoxOp_SecondOrderCFL.H:207-209).

Here rank r owns the radial cells [lo, hi) of all six panels, so panel seams
and their flux register never cross ranks, and its level holds `halo` more
radial layers on each side that has a neighbour.  Before each RK4 stage the
rank receives those layers of the stage state from its neighbours (the
layers they own next to the boundary) and then runs the stage on its whole
level.  The owned cells come out bit-identical to the single-level step:

* every value an owned cell's update reads lies within `halo` radial layers
  of it (order 2: the stage primitives, 2 layers; order 4: the operator
  reads 5 ghost layers of native averages, each made from the stage state
  within 1 radial cell, so 6);
* the slab's metric tables use the shell's radial index and spacing
  (`Params.radial_offset`, `Params.radial_cells`);
* the CFL rate is a maximum, taken after the exchange, so the maximum over
  ranks is the shell's exactly.

The halo layers' own updates are replaced at the next exchange, so at order
4 the operator runs on the owned layers only (`Shell.set_radial_window`) and
the halo costs only its share of the stage preparation; `owned()` returns
the layers a rank is responsible for.
The exchange is point-to-point between radial neighbours (NCCL between
GPUs, gloo between host processes); the dt reduction is one all-reduce.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import torch

from .level import Params

HALO = {2: 2, 4: 6}


def slab_range(nr: int, world: int, rank: int) -> tuple[int, int]:
    """Radial cells [lo, hi) rank `rank` owns: sizes differ by at most one."""
    return rank * nr // world, (rank + 1) * nr // world


@dataclass(frozen=True)
class SlabPlan:
    """Which radial layers rank `rank` of `world` owns, holds and swaps."""
    nr: int
    world: int
    rank: int
    halo: int

    def __post_init__(self):
        if not 0 <= self.rank < self.world:
            raise ValueError(f"rank {self.rank} outside a world of {self.world}")
        if self.nr // self.world < max(self.halo, 4):
            raise ValueError(f"{self.world} slabs of a {self.nr}-cell shell own fewer than "
                             f"max(halo {self.halo}, 4) radial cells each")

    @property
    def lo(self) -> int:
        return slab_range(self.nr, self.world, self.rank)[0]

    @property
    def hi(self) -> int:
        return slab_range(self.nr, self.world, self.rank)[1]

    @property
    def below(self) -> int:
        return self.halo if self.rank > 0 else 0

    @property
    def above(self) -> int:
        return self.halo if self.rank < self.world - 1 else 0

    @property
    def local_nr(self) -> int:
        return self.hi - self.lo + self.below + self.above

    @property
    def offset(self) -> int:
        return self.lo - self.below

    def params(self, shell: Params) -> Params:
        if shell.radial_cells or shell.radial_offset:
            raise ValueError("the shell to split must be a whole shell")
        return replace(shell, nr=self.local_nr, radial_offset=self.offset, radial_cells=self.nr)

    def links(self, first: int) -> list[tuple[int, slice, slice]]:
        """(neighbour rank, columns sent to it, columns received from it) of a
        (rows, radial) view whose first level cell is at column `first`."""
        own, b, h = self.hi - self.lo, self.below, self.halo
        out = []
        if self.rank > 0:
            out.append((self.rank - 1, slice(first + b, first + b + h), slice(first, first + b)))
        if self.rank < self.world - 1:
            out.append((self.rank + 1, slice(first + b + own - h, first + b + own),
                        slice(first + b + own, first + b + own + self.above)))
        return out


class LocalTransport:
    """All slabs in this process (one GPU, or the host): halo layers move by
    copies between their buffers."""

    def exchange(self, plans: list[SlabPlan], bufs: list[tuple[torch.Tensor, int]]) -> None:
        at = {p.rank: q for q, p in enumerate(plans)}
        for q, plan in enumerate(plans):
            buf, first = bufs[q]
            for peer, send, _ in plan.links(first):
                dst, dfirst = bufs[at[peer]]
                recv = next(r for p, _, r in plans[at[peer]].links(dfirst) if p == plan.rank)
                dst[:, recv].copy_(buf[:, send])

    def max(self, values: list[torch.Tensor]) -> torch.Tensor:
        out = values[0].clone()
        for v in values[1:]:
            torch.maximum(out, v, out=out)
        return out

    def collect(self, plans: list[SlabPlan], owned: list[torch.Tensor]) -> torch.Tensor:
        return torch.cat([owned[q] for q in sorted(range(len(plans)), key=lambda q: plans[q].rank)], dim=-1)

    def barrier(self) -> None:
        pass


class SlabExchangeError(RuntimeError):
    """A halo swap with a neighbouring rank failed (the rank left, or the
    process group's timeout ran out)."""


class DistTransport:
    """One slab per process: halo layers swap with the radial neighbours by
    torch.distributed point-to-point operations (NCCL between GPUs, gloo on
    the host), the CFL rate by an all-reduce of its maximum."""

    def __init__(self, group=None):
        self.group = group

    def exchange(self, plans: list[SlabPlan], bufs: list[tuple[torch.Tensor, int]]) -> None:
        import torch.distributed as dist
        (plan,), ((buf, first),) = plans, bufs
        ops, landing = [], []
        for peer, send, recv in plan.links(first):
            ops.append(dist.P2POp(dist.isend, buf[:, send].contiguous(), peer, self.group))
            tmp = torch.empty((buf.shape[0], recv.stop - recv.start), dtype=buf.dtype, device=buf.device)
            ops.append(dist.P2POp(dist.irecv, tmp, peer, self.group))
            landing.append((recv, tmp))
        if ops:
            try:
                for work in dist.batch_isend_irecv(ops):
                    work.wait()
            except RuntimeError as e:
                # a neighbour that left (or timed out) ends the swap with an
                # error instead of a wait
                peers = [p for p, _, _ in plan.links(first)]
                raise SlabExchangeError(f"rank {plan.rank}: halo swap with ranks {peers} failed: {e}") from e
        for recv, tmp in landing:
            buf[:, recv].copy_(tmp)

    def agree(self, key: list[int]) -> None:
        """Raise ValueError on every rank unless every rank passes the same
        key (one all-gather): ranks that split different shells would swap
        halo buffers of different shapes."""
        import torch.distributed as dist
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(self.group) == "nccl" else "cpu"
        mine = torch.tensor(key, dtype=torch.int64, device=dev)
        every = [torch.empty_like(mine) for _ in range(dist.get_world_size(self.group))]
        dist.all_gather(every, mine, group=self.group)
        bad = [r for r, k in enumerate(every) if not torch.equal(k, mine)]
        if bad:
            raise ValueError(f"ranks {bad} split a different shell (parameters or world size differ)")

    def max(self, values: list[torch.Tensor]) -> torch.Tensor:
        import torch.distributed as dist
        (v,) = values
        out = v.clone()
        dist.all_reduce(out, op=dist.ReduceOp.MAX, group=self.group)
        return out

    def collect(self, plans: list[SlabPlan], owned: list[torch.Tensor]) -> torch.Tensor | None:
        """The whole shell's cells on rank 0 (None on the others): every
        rank sends rank 0 the cells it owns."""
        import torch.distributed as dist
        (plan,), (mine,) = plans, owned
        mine = mine.contiguous()
        if plan.rank != 0:
            dist.send(mine, 0, group=self.group)
            return None
        parts = [mine]
        for r in range(1, plan.world):
            lo, hi = slab_range(plan.nr, plan.world, r)
            part = torch.empty(mine.shape[:-1] + (hi - lo,), dtype=mine.dtype, device=mine.device)
            dist.recv(part, r, group=self.group)
            parts.append(part)
        return torch.cat(parts, dim=-1)

    def barrier(self) -> None:
        import torch.distributed as dist
        dist.barrier(group=self.group)


def _fingerprint(params: Params, world: int, halo: int) -> list[int]:
    """Integers that differ when two ranks would split different shells:
    the options, the bit patterns of the real parameters, world and halo."""
    import struct
    key = [world, halo]
    for _, v in sorted(vars(params).items()):
        key.append(struct.unpack("<q", struct.pack("<d", float(v)))[0] if isinstance(v, float) else int(v))
    return key


class ShardedShell:
    """The slabs of one shell that this process drives: its own under
    torch.distributed (`ShardedShell(params, rank, world)`), or every slab on
    one device (`ShardedShell.emulated(params, world)`).

    Methods take and return one state per local slab, each a level state of
    the slab (level layout, `local_nr` radial cells)."""

    def __init__(self, params: Params, rank: int, world: int, transport=None, device: int | None = None,
                 level=None, halo: int | None = None, ranks: list[int] | None = None):
        from .level import Shell
        halo = HALO[params.spatial_order] if halo is None else halo
        self.params = params
        self.world = world
        self.plans = [SlabPlan(params.nr, world, r, halo) for r in (ranks if ranks is not None else [rank])]
        if len(self.plans) not in (1, world) or len({p.rank for p in self.plans}) != len(self.plans):
            raise ValueError("a process drives its own slab or every slab of the shell once")
        if transport is None:
            transport = DistTransport() if world > 1 and len(self.plans) == 1 else LocalTransport()
        self.transport = transport
        if hasattr(transport, "agree"):
            transport.agree(_fingerprint(params, world, halo))
        make = level if level is not None else (lambda p: Shell(p, device))
        self.levels = [make(plan.params(params)) for plan in self.plans]
        if params.spatial_order == 4 and world > 1:
            # the halo layers' rhs is never used: the operator runs on the
            # owned layers only (the stage preparation still covers the slab)
            for plan, lvl in zip(self.plans, self.levels):
                if hasattr(lvl, "set_radial_window"):
                    lvl.set_radial_window(plan.below, plan.below + plan.hi - plan.lo)

    @classmethod
    def emulated(cls, params: Params, world: int, device: int | None = None, level=None,
                 halo: int | None = None) -> "ShardedShell":
        return cls(params, 0, world, LocalTransport(), device, level, halo, ranks=list(range(world)))

    def close(self) -> None:
        for lvl in self.levels:
            if hasattr(lvl, "close"):
                lvl.close()
        self.levels = []

    def new_states(self) -> list[torch.Tensor]:
        return [lvl.new_state() for lvl in self.levels]

    def _shape(self, plan: SlabPlan) -> tuple[int, ...]:
        na = self.params.na
        return 6, 8, na, na, plan.local_nr

    def scatter(self, full: torch.Tensor) -> list[torch.Tensor]:
        """Each local slab's state (halo layers included) from a whole-shell
        state (level layout of the whole shell, on any device)."""
        na, nr = self.params.na, self.params.nr
        f = full.reshape(6, 8, na, na, nr)
        out = []
        for plan, lvl in zip(self.plans, self.levels):
            st = lvl.new_state()
            st.view(self._shape(plan)).copy_(f[..., plan.offset:plan.offset + plan.local_nr])
            out.append(st)
        return out

    def owned(self, states: list[torch.Tensor]) -> list[torch.Tensor]:
        """Views of the radial cells each local slab owns, (6, 8, na, na, hi - lo)."""
        return [st.view(self._shape(p))[..., p.below:p.below + p.hi - p.lo] for p, st in zip(self.plans, states)]

    def gather(self, states: list[torch.Tensor]) -> torch.Tensor:
        """The whole-shell state from the local slabs (emulated slabs only)."""
        if len(self.plans) != self.world:
            raise ValueError("gather needs every slab in this process")
        return torch.cat(self.owned(states), dim=-1)

    def save(self, path: str, states: list[torch.Tensor], time: float, step: int = 0,
             attributes: dict | None = None) -> None:
        """Write the shell as one whole-shell checkpoint
        (heliocubed_b200.checkpoint, the format a single-GPU level reads):
        rank 0 collects the cells every rank owns and writes the file; every
        rank returns once it is written."""
        from . import checkpoint
        full = self.transport.collect(self.plans, self.owned(states))
        if full is not None:
            checkpoint.save(path, self.params, full, time, step, attributes)
        self.transport.barrier()

    def load(self, path: str) -> tuple[list[torch.Tensor], float, int, dict]:
        """Each local slab's state (halo layers included) from a whole-shell
        checkpoint of this shell: (states, time, step, attributes)."""
        from . import checkpoint
        params, state, time, step, attributes = checkpoint.load(path)
        if params != self.params:
            raise checkpoint.CheckpointError(f"{path}: a checkpoint of another shell")
        return self.scatter(torch.from_numpy(state)), time, step, attributes

    def exchange(self, states: list[torch.Tensor], stage: int) -> None:
        """Halo layers of the buffer stage `stage` reads, from the neighbours."""
        if self.world > 1:
            self.transport.exchange(self.plans, [lvl.stage_state(st, stage) for lvl, st in zip(self.levels, states)])

    def inv_dt_max(self, states: list[torch.Tensor]) -> torch.Tensor:
        """The shell's maximum CFL rate (one element, on the slabs' device);
        refreshes the halo layers of the states first."""
        self.exchange(states, 0)
        return self.transport.max([lvl.inv_dt_max(st) for lvl, st in zip(self.levels, states)])

    def rk4_step(self, states: list[torch.Tensor], dt: float, t: float = 0.0) -> None:
        """One RK4 step of the shell with dt from the host."""
        for stage in range(4):
            self.exchange(states, stage)
            for lvl, st in zip(self.levels, states):
                lvl.rk4_stage(st, stage, dt, t)

    def advance(self, states: list[torch.Tensor], nsteps: int, time: torch.Tensor) -> None:
        """nsteps RK4 steps with dt = cfl / (the shell's maximum CFL rate),
        kept on the device: no host synchronisation between steps.  `time`
        (one element, device) advances by each step's dt."""
        for _ in range(nsteps):
            inv = self.inv_dt_max(states)
            for stage in range(4):
                if stage:
                    self.exchange(states, stage)
                for lvl, st in zip(self.levels, states):
                    lvl.rk4_stage(st, stage, inv_dt=inv, time=time)
            # cfl / inv as one division (a float over a tensor would take
            # its reciprocal and multiply, one rounding more than the stages')
            time += torch.full_like(inv, self.params.cfl) / inv
