"""Served ensemble of cubed-sphere MHD solves on one GPU.

A request is one solve: a six-panel shell of its own size and scheme (second
order PLM-MC + Rusanov, or fourth order Berta WENOZ + Roe), the cone-CME
cloud of its parameters inserted on the device at admission into the
ambient wind, and a number of RK4 steps with dt from the device CFL
reduction.  The server keeps every admitted
state resident in HBM and overlaps requests on the GPU:

* admission: requests are admitted in arrival order while the HBM estimate
  of the admitted solves stays under the budget and fewer than `max_inflight`
  run; a solve that finishes frees its slot for the next arrival at once
  (continuous batching: new requests join while others are mid-flight);
* slots: a slot is a level context (geometry tables and stage workspace),
  its state buffer, its own CUDA stream and a CUDA graph of `chunk`
  hc_level_advance_cfl steps captured on that buffer; slots are pooled by
  shape and reused, so admission costs two kernels (wind, cone insertion)
  on the slot's stream, not a context build;
* progress: every slot whose previous chunk has completed gets its next
  chunk; the GPU runs the chunks of different slots concurrently;
* fourth-order cohort (cobatch=True): the fourth-order requests in flight,
  whatever their sizes, step together as one ensemble (hc_ensemble): each
  keeps its own state, CFL dt, model time and insertion schedule, and each
  kernel of the stage operator is one launch over all their panels.  The
  cohort advances in chunks of min(chunk, fewest steps left) steps on its
  own stream; between chunks finished requests leave (their results are
  copied out) and newly admitted ones join.

`run_plain` is the drop-in path beside it: the same requests one after
another, each through the eager per-solve launches of `Shell.advance`.
Results are identical in both: the kernels are deterministic (the CFL max is
order independent) and every slot owns its buffers.
"""
from __future__ import annotations

import hashlib
import time
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .level import ConeSpec, Ensemble, InitSpec, Params, Shell, prepare_cone


@dataclass
class Cone:
    """Cone-CME parameters of a request: a finite spherical cloud (the
    reference's cone field model 4, ConeSpec) of `density_ratio` times the
    wind's density at the inner boundary, moving radially at `speed_kms`,
    its axis at (lat, lon) and its radius r_inner sin(half width).  The cloud
    lies wholly in the shell, touching the inner boundary, when it is
    inserted on the device at admission (hc_level_insert_cone)."""
    speed_kms: float = 1000.0
    half_width_deg: float = 30.0
    lat_deg: float = 0.0
    lon_deg: float = 0.0
    density_ratio: float = 4.0
    temperature: float = 1.0e6

    def prepared(self, params: Params, wind: InitSpec | None = None) -> N.HcCone:
        wind = wind or wind_spec()
        rho_inner = wind.rho0 * (wind.r_ref / params.inner_radius) ** 2
        spec = ConeSpec.on_inner_boundary(params.inner_radius, lat_deg=self.lat_deg, lon_deg=self.lon_deg,
                                          half_angle_deg=self.half_width_deg, apex_speed=self.speed_kms,
                                          density=self.density_ratio * rho_inner, temperature=self.temperature)
        return prepare_cone(spec, params.inner_radius)


def wind_spec() -> InitSpec:
    """The ambient state of every request: the Parker-like wind of InitSpec
    without its pressure pulse."""
    return InitSpec(pulse_amp=0.0)


@dataclass
class Request:
    rid: int
    nr: int
    na: int
    order: int
    steps: int
    arrival: float = 0.0      # seconds after the start of the run
    cone: Cone = field(default_factory=Cone)
    # Optional initial state from the host (pinned float64, the level's JU
    # layout), e.g. a restart: copied to the device at admission in place of
    # the on-device wind and cone insertion; the cone still sets the
    # insertion schedule and the model time.
    initial: "torch.Tensor | None" = None

    @property
    def cells(self) -> int:
        return 6 * self.nr * self.na * self.na

    def params(self) -> Params:
        if self.order == 4:
            return Params(nr=self.nr, na=self.na, spatial_order=4, riemann_solver=2, berta_fallback_type=0,
                          autotune=1)
        return Params(nr=self.nr, na=self.na, spatial_order=2, limiter=3, riemann_solver=1, autotune=1)


def admit(shell: Shell, req: Request, ju: torch.Tensor, time_dev: torch.Tensor, schedule: bool = True) -> None:
    """Device-side admission on the current stream: the wind into `ju`, the
    request's cone cloud inserted at its insertion time, the model time set
    to that time, and the insertion schedule (CFL ramp, and the Rusanov
    window of fourth-order Roe solves) that the reference's driver applies
    after an insertion (schedule=False: the state only)."""
    cone = req.cone.prepared(shell.params)
    if req.initial is not None:
        ju.copy_(req.initial, non_blocking=True)
    else:
        shell.init(wind_spec(), ju)
        shell.insert_cone(cone, cone.insertion_time, ju)
    if schedule:
        shell.set_cme_schedule([cone])
    time_dev.fill_(cone.insertion_time)


def initial_state(shell: Shell, req: Request) -> np.ndarray:
    """Host copy of the state `admit` builds from the request's parameters
    (for checks, reports and host-staged requests); the shell's insertion
    schedule is left as it was."""
    ju = shell.new_state()
    t = torch.zeros(1, dtype=torch.float64, device=ju.device)
    params_only = Request(req.rid, req.nr, req.na, req.order, req.steps, req.arrival, req.cone)
    admit(shell, params_only, ju, t, schedule=False)
    return ju.cpu().numpy()


def fingerprint(state: torch.Tensor, out: torch.Tensor) -> None:
    """Enqueue on the current stream a bitwise fingerprint of a float64
    state into out[0:4] (int64 on the device): the sums, modulo 2^64, of the
    bit patterns of all values, of every second and of every third value,
    and the count of non-finite values.  Integer sums do not depend on the
    reduction order, so equal states give equal fingerprints and any changed
    bit changes the first sum."""
    bits = state.view(torch.int64)
    out[0] = bits.sum()
    out[1] = bits[1::2].sum()
    out[2] = bits[::3].sum()
    out[3] = torch.isfinite(state).logical_not().sum()


class Slot:
    """A pooled level context with its state buffer, stream and step graph
    (graph=False: no graph, for slots that step in a cohort)."""

    def __init__(self, shape: tuple[int, int, int], chunk: int, device: int, graph: bool = True):
        nr, na, order = shape
        free0 = torch.cuda.mem_get_info(device)[0]
        self.shape = shape
        self.chunk = chunk
        self.shell = Shell(Request(0, nr, na, order, 0).params(), device=device)
        self.stream = torch.cuda.Stream(device=device)
        self.state = self.shell.new_state()
        self.time = torch.zeros(1, dtype=torch.float64, device=self.shell._dev)
        self.host_out = torch.empty(self.state.numel(), dtype=torch.float64).pin_memory()
        self.host_time = torch.empty(1, dtype=torch.float64).pin_memory()
        self.print_dev = torch.zeros(4, dtype=torch.int64, device=self.shell._dev)
        self.host_print = torch.zeros(4, dtype=torch.int64).pin_memory()
        self.fingerprint = False  # set by the server: results as fingerprints
        # capture on a valid (wind) state with the (empty) insertion schedule
        # in the step; admission overwrites the buffer and the schedule
        self.shell.init(wind_spec(), self.state)
        self.shell.set_cme_schedule([])
        torch.cuda.synchronize(device)
        with torch.cuda.stream(self.stream):
            if graph:
                self.graph = self.shell.capture_advance(self.state, chunk, self.time)
            else:
                # one eager step builds the stage buffers (and tunes) now
                self.graph = None
                self.shell.advance(self.state, 1, self.time)
        torch.cuda.synchronize(device)
        self.bytes = max(0, free0 - torch.cuda.mem_get_info(device)[0])
        self.req: Request | None = None
        self.left = 0
        self.event: torch.cuda.Event | None = None
        self.t_start = 0.0
        self.in_cohort = False

    def start(self, req: Request, now: float) -> None:
        self.req = req
        self.left = req.steps
        self.t_start = now
        with torch.cuda.stream(self.stream):
            admit(self.shell, req, self.state, self.time)
        self.event = None

    def issue(self) -> None:
        """Enqueue the next chunk (a graph replay, or the eager remainder);
        with no steps left, the copy of the result to the host."""
        with torch.cuda.stream(self.stream):
            if self.left >= self.chunk and self.graph is not None:
                self.graph.replay()
                self.left -= self.chunk
            elif self.left > 0:
                steps = self.left if self.graph is not None else min(self.left, self.chunk)
                self.shell.advance(self.state, steps, self.time)
                self.left -= steps
            else:
                self.host_out.copy_(self.state, non_blocking=True)
                self.host_time.copy_(self.time, non_blocking=True)
                if self.fingerprint:
                    fingerprint(self.state, self.print_dev)
                    self.host_print.copy_(self.print_dev, non_blocking=True)
                self.left = -1
            self.event = torch.cuda.Event()
            self.event.record(self.stream)


class Cohort:
    """The fourth-order slots in flight, stepped together as an ensemble on
    one stream (see the module docstring).  Ensembles are kept by their
    member slots (slots are pooled, so a membership can recur), the
    `max_kept` most recently used ones: releasing one frees device memory,
    which synchronises the GPU, so it happens only between chunks and only
    past that count.  The device calls go through the methods at the end of
    the class."""

    max_kept = 512

    def __init__(self, chunk: int, device: int):
        self.chunk = chunk
        self.device = device
        self.stream = self._new_stream()
        self.members: list[Slot] = []
        self.joining: list[tuple[Slot, object]] = []
        self.event = None
        self.ensembles: "OrderedDict[tuple[int, ...], object]" = OrderedDict()
        self.chunk_steps = 0  # steps of all launched chunks (each step: one operator launch group per stage)

    def join(self, slot: Slot) -> None:
        """Take an admitted slot (its admission is on the slot's stream)."""
        slot.in_cohort = True
        self.joining.append((slot, self._record(slot.stream)))

    def progress(self) -> bool:
        """Once the running chunk has completed: hand finished members their
        result copy, take in the joining slots and launch the next chunk.
        True when anything was done."""
        if self.event is not None and not self.event.query():
            return False
        if not self.members and not self.joining:
            return False
        for slot in [s for s in self.members if s.left == 0]:
            self._wait(slot.stream, self.event)
            slot.in_cohort = False
            slot.issue()  # the copy of the result, on the slot's own stream
        self.members = [s for s in self.members if s.left > 0]
        for slot, admitted in self.joining:
            self._wait(self.stream, admitted)
            self.members.append(slot)
        self.joining = []
        self.event = None
        if not self.members:
            return True
        steps = min(self.chunk, min(s.left for s in self.members))
        key = tuple(id(s) for s in self.members)
        ens = self.ensembles.get(key)
        if ens is None:
            ens = self.ensembles[key] = self._ensemble(self.members)
            while len(self.ensembles) > self.max_kept:
                self.ensembles.popitem(last=False)[1].close()
        else:
            self.ensembles.move_to_end(key)
        self._advance(ens, self.members, steps)
        self.chunk_steps += steps
        for s in self.members:
            s.left -= steps
        self.event = self._record(self.stream)
        return True

    def close(self) -> None:
        for ens in self.ensembles.values():
            ens.close()
        self.ensembles.clear()

    # device calls
    def _new_stream(self):
        return torch.cuda.Stream(device=self.device)

    @staticmethod
    def _record(stream):
        ev = torch.cuda.Event()
        ev.record(stream)
        return ev

    @staticmethod
    def _wait(stream, event) -> None:
        stream.wait_event(event)

    @staticmethod
    def _ensemble(slots: list[Slot]):
        return Ensemble([s.shell for s in slots])

    def _advance(self, ens, slots: list[Slot], steps: int) -> None:
        with torch.cuda.stream(self.stream):
            ens.advance([s.state for s in slots], steps, [s.time for s in slots])


@dataclass
class Result:
    rid: int
    cells: int
    steps: int
    t_arrival: float
    t_start: float
    t_done: float
    state: np.ndarray
    model_time: float
    error: str | None = None   # set (and state empty) when the request was refused
    # with keep_states=False: the state's fingerprint (see fingerprint()) and
    # finiteness instead of the state itself (state empty); the state is still
    # copied to the host
    digest: bytes | None = None
    finite: bool | None = None

    @property
    def time_to_solution(self) -> float:
        return self.t_done - self.t_arrival


class EnsembleServer:
    """Continuous-batching server over pooled slots (see module docstring)."""

    def __init__(self, hbm_budget: float, max_inflight: int = 8, chunk: int = 10, device: int | None = None,
                 keep_states: bool = True, cobatch: bool = True):
        self.keep_states = keep_states
        self.cobatch = cobatch
        self.budget = hbm_budget
        self.max_inflight = max_inflight
        self.chunk = chunk
        self.device = torch.cuda.current_device() if device is None else device
        self.pool: dict[tuple, list[Slot]] = {}
        self.slot_bytes: dict[tuple, int] = {}
        self.in_use = 0.0
        self.cohort: Cohort | None = None  # built when the first fourth-order request joins

    @staticmethod
    def shape(req: Request) -> tuple[int, int, int]:
        return (req.nr, req.na, req.order)

    def warm(self, requests: list[Request], per_shape: int = 1) -> None:
        """Build slots ahead of time (contexts, buffers, graphs)."""
        for shp in sorted({self.shape(r) for r in requests}):
            for _ in range(per_shape - len(self.pool.get(shp, []))):
                s = self._new_slot(shp)
                self.pool.setdefault(shp, []).append(s)
                self.slot_bytes[shp] = s.bytes

    # Device bytes per cell of a slot of each order before any slot of that
    # order was built (state, stage workspace, operator scratch and the
    # graph's pool; generous, so an unseen shape is not admitted past the
    # budget).  Measured slots replace it.
    BYTES_PER_CELL_GUESS = {2: 64 * 8, 4: 64 * 40}

    def estimate_bytes(self, shp: tuple[int, int, int]) -> int:
        """HBM a slot of shape `shp` takes: its measured size, else the
        largest measured bytes per cell of a slot of the same order times its
        cells, else a fixed guess per cell."""
        if shp in self.slot_bytes:
            return self.slot_bytes[shp]
        nr, na, order = shp
        cells = 6 * nr * na * na
        per_cell = [b / (6 * s[0] * s[1] * s[1]) for s, b in self.slot_bytes.items() if s[2] == order]
        return int(cells * (max(per_cell) if per_cell else self.BYTES_PER_CELL_GUESS.get(order, 64 * 40)))

    def _new_slot(self, shp: tuple[int, int, int]) -> Slot:
        return Slot(shp, self.chunk, self.device, graph=not (self.cobatch and shp[2] == 4))

    def _acquire(self, req: Request) -> Slot | None:
        shp = self.shape(req)
        need = self.estimate_bytes(shp)
        if self.in_use + need > self.budget:
            return None
        idle = self.pool.setdefault(shp, [])
        slot = idle.pop() if idle else self._new_slot(shp)
        self.slot_bytes[shp] = max(self.slot_bytes.get(shp, 0), slot.bytes)
        self.in_use += self.slot_bytes[shp]
        return slot

    def _release(self, slot: Slot) -> None:
        self.in_use -= self.slot_bytes[slot.shape]
        slot.req = None
        self.pool[slot.shape].append(slot)

    def run(self, requests: list[Request]) -> list[Result]:
        """Serve `requests` (arrival times relative to the call)."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active: list[Slot] = []
        results: list[Result] = []
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_inflight:
                slot = self._acquire(pending[0])
                if slot is None:
                    if not active:
                        # nothing runs, so nothing will free memory: the
                        # request alone needs more than the whole budget
                        req = pending.pop(0)
                        need = self.estimate_bytes(self.shape(req))
                        results.append(Result(req.rid, req.cells, req.steps, req.arrival, now, now,
                                              np.empty(0), float("nan"),
                                              error=f"request needs {need} B of HBM, over the budget of "
                                                    f"{self.budget:.0f} B"))
                        continue
                    break
                req = pending.pop(0)
                slot.fingerprint = not self.keep_states
                slot.start(req, now)
                if self.cobatch and req.order == 4 and req.steps > 0:
                    if self.cohort is None:
                        self.cohort = Cohort(self.chunk, self.device)
                    self.cohort.join(slot)
                else:
                    slot.issue()
                active.append(slot)
            progressed = self.cohort.progress() if self.cohort is not None else False
            for slot in list(active):
                if slot.in_cohort:
                    continue
                if slot.event is not None and not slot.event.query():
                    continue
                progressed = True
                if slot.left == -1:
                    req = slot.req
                    results.append(_result(req, slot.t_start, time.perf_counter() - t0, slot.host_out.numpy(),
                                           float(slot.host_time.item()), self.keep_states,
                                           slot.host_print.numpy() if slot.fingerprint else None))
                    active.remove(slot)
                    self._release(slot)
                else:
                    slot.issue()
            if not progressed:
                if active:
                    time.sleep(2e-5)
                elif pending:
                    time.sleep(max(0.0, min(1e-3, pending[0].arrival - (time.perf_counter() - t0))))
        return results


    def forget_ensembles(self) -> None:
        """Release the cohort's cached ensembles (between runs: the next run
        builds its memberships anew, as the first one did).  Frees device
        memory, which synchronises the GPU."""
        if self.cohort is not None:
            self.cohort.close()

    def close(self) -> None:
        """Release every pooled slot (contexts, buffers, graphs) and the
        cohort's ensembles."""
        if self.cohort is not None:
            self.cohort.close()
        for slots in self.pool.values():
            for slot in slots:
                slot.graph = None
                slot.shell.close()
        self.pool.clear()


def _result(req: Request, t_start: float, t_done: float, host_state: np.ndarray, model_time: float,
            keep: bool, prints: np.ndarray | None = None) -> Result:
    if keep:
        return Result(req.rid, req.cells, req.steps, req.arrival, t_start, t_done, host_state.copy(), model_time)
    if prints is None:  # no device fingerprint: hash the host copy
        return Result(req.rid, req.cells, req.steps, req.arrival, t_start, t_done, np.empty(0), model_time,
                      digest=hashlib.sha256(host_state.tobytes()).digest(),
                      finite=bool(np.isfinite(host_state).all()))
    return Result(req.rid, req.cells, req.steps, req.arrival, t_start, t_done, np.empty(0), model_time,
                  digest=prints[:3].tobytes(), finite=bool(prints[3] == 0))


def same_results(a: list[Result], b: list[Result]) -> bool:
    """Bit-identical final states of the same requests in two runs (states or
    digests, NaN patterns included)."""
    if len(a) != len(b):
        return False
    for x, y in zip(sorted(a, key=lambda r: r.rid), sorted(b, key=lambda r: r.rid)):
        if x.rid != y.rid:
            return False
        if x.digest is not None or y.digest is not None:
            if x.digest != y.digest:
                return False
        elif not np.array_equal(x.state, y.state, equal_nan=True):
            return False
    return True


def run_plain(requests: list[Request], device: int | None = None,
              shells: dict[tuple, Shell] | None = None, keep_states: bool = True) -> list[Result]:
    """The same requests one after another through eager per-solve launches
    (`admit`, `Shell.advance`, the result copied to the host); contexts are
    cached by shape so neither path pays for context builds."""
    device = torch.cuda.current_device() if device is None else device
    shells = {} if shells is None else shells
    results = []
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        wait = req.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        shp = (req.nr, req.na, req.order)
        if shp not in shells:
            shells[shp] = Shell(req.params(), device=device)
        sh = shells[shp]
        t_start = time.perf_counter() - t0
        ju = sh.new_state()
        t = torch.zeros(1, dtype=torch.float64, device=sh._dev)
        admit(sh, req, ju, t)
        sh.advance(ju, req.steps, t)
        prints = None
        if not keep_states:
            pd = torch.zeros(4, dtype=torch.int64, device=sh._dev)
            fingerprint(ju, pd)
            prints = pd.cpu().numpy()
        out = ju.cpu().numpy()
        results.append(_result(req, t_start, time.perf_counter() - t0, out, float(t.item()), keep_states, prints))
    return results


def synthetic_requests(n: int, seed: int, rate_hz: float | None, steps: int,
                       radial=(32, 48, 64, 96), angular=(32, 48, 64), orders=(2, 4)) -> list[Request]:
    """Seeded requests: grid from `radial` x `angular`^2, scheme 50/50 from
    `orders`, cone speed U[500, 2000] km/s, half-width U[20, 60] deg,
    lat/lon U[-30, 30] deg, density ratio U[2, 6]; Poisson arrivals at
    `rate_hz` (all at t = 0 when None).  The arrival times come from their
    own stream, so the requests themselves do not depend on the rate."""
    rng = np.random.default_rng(seed)
    arrivals = np.random.default_rng([seed, 1])
    t = 0.0
    out = []
    for rid in range(n):
        if rate_hz:
            t += arrivals.exponential(1.0 / rate_hz)
        cone = Cone(speed_kms=rng.uniform(500, 2000), half_width_deg=rng.uniform(20, 60),
                    lat_deg=rng.uniform(-30, 30), lon_deg=rng.uniform(-30, 30), density_ratio=rng.uniform(2, 6))
        out.append(Request(rid, int(rng.choice(radial)), int(rng.choice(angular)), int(rng.choice(orders)), steps,
                           t if rate_hz else 0.0, cone))
    return out


def summarize(results: list[Result]) -> dict:
    results = [r for r in results if r.error is None]
    tts = np.array([r.time_to_solution for r in results])
    span = max(r.t_done for r in results) - min(r.t_arrival for r in results)
    work = sum(r.cells * r.steps for r in results)
    return {"requests": len(results), "cell_updates": work, "makespan_s": span,
            "cell_updates_per_s": work / span, "p50_s": float(np.percentile(tts, 50)),
            "p99_s": float(np.percentile(tts, 99))}
