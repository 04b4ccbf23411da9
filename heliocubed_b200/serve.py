"""Served ensemble of cubed-sphere MHD solves on one GPU.

A request is one solve: a six-panel shell of its own size and scheme (second
order PLM-MC + Rusanov, or fourth order Berta WENOZ + Roe), a synthetic
cone-shaped plasma cloud inserted at admission, and a number of RK4 steps
with dt from the device CFL reduction.  The server keeps every admitted
state resident in HBM and overlaps requests on the GPU:

* admission: requests are admitted in arrival order while the HBM estimate
  of the admitted solves stays under the budget and fewer than `max_inflight`
  run; a solve that finishes frees its slot for the next arrival at once
  (continuous batching: new requests join while others are mid-flight);
* slots: a slot is a level context (geometry tables and stage workspace),
  its state buffer, its own CUDA stream and a CUDA graph of `chunk`
  hc_level_advance_cfl steps captured on that buffer; slots are pooled by
  shape and reused, so admission costs a host-to-device copy, not a context
  build;
* progress: every slot whose previous chunk has completed gets its next
  chunk; the GPU runs the chunks of different slots concurrently.

`run_plain` is the drop-in path beside it: the same requests one after
another, each through the eager per-solve launches of `Shell.advance`.
Results are identical in both: the kernels are deterministic (the CFL max is
order independent) and every slot owns its buffers.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .level import C_SR, InitSpec, Params, Shell, cell_directions


@dataclass
class Cone:
    """Synthetic cone-shaped cloud: inside `half_width_deg` of the axis at
    (lat, lon) and below `r_top` (cm), the density is `density_ratio` times
    the wind's and the radial speed `speed_kms`; pressure and field are the
    wind's.  The edges are tapered smoothly (cos^2 over +-`edge` of the half
    width and of r_top): a sharp-edged cloud moving at up to 2000 km/s
    through the 400 km/s wind is a discontinuous initial state that the
    fourth-order scheme need not survive at coarse grids."""
    speed_kms: float = 1000.0
    half_width_deg: float = 30.0
    lat_deg: float = 0.0
    lon_deg: float = 0.0
    density_ratio: float = 4.0
    r_top: float = 30.0 * C_SR
    edge: float = 0.25


@dataclass
class Request:
    rid: int
    nr: int
    na: int
    order: int
    steps: int
    arrival: float = 0.0      # seconds after the start of the run
    cone: Cone = field(default_factory=Cone)

    @property
    def cells(self) -> int:
        return 6 * self.nr * self.na * self.na

    def params(self) -> Params:
        if self.order == 4:
            return Params(nr=self.nr, na=self.na, spatial_order=4, riemann_solver=2, berta_fallback_type=0)
        return Params(nr=self.nr, na=self.na, spatial_order=2, limiter=3, riemann_solver=1)


def cone_state(params: Params, det: np.ndarray, dvolr: np.ndarray, cone: Cone,
               spec: InitSpec | None = None) -> np.ndarray:
    """JU [6][8][k][j][i] of the Parker-like wind of InitSpec with the cone
    cloud; cell averages as J x centre values (J = <det A> dVolr)."""
    spec = spec or InitSpec()
    nr, na, gam = params.nr, params.na, params.gamma
    r0, r1, C = params.inner_radius, params.outer_radius, params.radial_stretch
    Rt = (r1 - r0) / np.expm1(C)
    r = r0 + Rt * np.expm1(C * (np.arange(nr) + 0.5) / nr)
    s = spec.r_ref / r
    X = cell_directions(na)                                      # [6][3][k][j]
    lat, lon = math.radians(cone.lat_deg), math.radians(cone.lon_deg)
    axis = np.array([math.cos(lat) * math.cos(lon), math.cos(lat) * math.sin(lon), math.sin(lat)])
    def taper(x, x0, width):
        """1 below x0 - width, 0 above x0 + width, cos^2 in between."""
        t = np.clip((x - (x0 - width)) / (2 * width), 0.0, 1.0)
        return np.cos(0.5 * np.pi * t) ** 2

    angle = np.arccos(np.clip(np.einsum("q,bqkj->bkj", axis, X), -1.0, 1.0))
    hw = math.radians(cone.half_width_deg)
    weight = taper(angle, hw, cone.edge * hw)[..., None] * taper(r, cone.r_top, cone.edge * (cone.r_top - r0))
    rho = spec.rho0 * s ** 2 * (1.0 + (cone.density_ratio - 1.0) * weight)
    vr = spec.vr + (cone.speed_kms * 1e5 - spec.vr) * weight
    p = spec.p0 * s ** (2 * gam) * np.ones_like(rho)
    Br = spec.b0 * s[None, None, None, :] ** 2 * np.sign(X[:, 2])[..., None]
    J = det[:, :, :, None] * dvolr[None, None, None, :]
    ju = np.zeros((6, 8, na, na, nr))
    v = vr[:, None] * X[..., None]
    B = Br[:, None] * X[..., None]
    ju[:, 0] = rho * J
    ju[:, 1:4] = rho[:, None] * v * J[:, None]
    ju[:, 5:8] = B * J[:, None]
    ju[:, 4] = (p / (gam - 1) + 0.5 * rho * (v ** 2).sum(1) + (B ** 2).sum(1) / (8 * np.pi)) * J
    return ju


def initial_state(shell: Shell, req: Request) -> np.ndarray:
    p = shell.params
    det = shell.geometry(4).reshape(6, p.na, p.na)
    dvolr = shell.geometry(0).reshape(p.nr + 1, 4)[:p.nr, 3]
    return np.ascontiguousarray(cone_state(p, det, dvolr, req.cone).reshape(-1))


class Slot:
    """A pooled level context with its state buffer, stream and step graph."""

    def __init__(self, shape: tuple[int, int, int], chunk: int, device: int):
        nr, na, order = shape
        free0 = torch.cuda.mem_get_info(device)[0]
        self.shape = shape
        self.chunk = chunk
        self.shell = Shell(Request(0, nr, na, order, 0).params(), device=device)
        self.stream = torch.cuda.Stream(device=device)
        self.state = self.shell.new_state()
        self.time = torch.zeros(1, dtype=torch.float64, device=self.shell._dev)
        self.host_in = torch.empty(self.state.numel(), dtype=torch.float64).pin_memory()
        self.host_out = torch.empty_like(self.host_in).pin_memory()
        self.host_time = torch.empty(1, dtype=torch.float64).pin_memory()
        # capture on a valid (wind) state; requests overwrite the buffer
        warm = Request(0, nr, na, order, 0, cone=Cone(density_ratio=1.0, speed_kms=400.0))
        self.state.copy_(torch.from_numpy(initial_state(self.shell, warm)).to(self.state.device))
        with torch.cuda.stream(self.stream):
            self.graph = self.shell.capture_advance(self.state, chunk, self.time)
        torch.cuda.synchronize(device)
        self.bytes = max(0, free0 - torch.cuda.mem_get_info(device)[0])
        self.req: Request | None = None
        self.left = 0
        self.event: torch.cuda.Event | None = None
        self.t_start = 0.0

    def start(self, req: Request, host_state: np.ndarray, now: float) -> None:
        self.req = req
        self.left = req.steps
        self.t_start = now
        self.host_in.numpy()[:] = host_state
        with torch.cuda.stream(self.stream):
            self.state.copy_(self.host_in, non_blocking=True)
            self.time.zero_()
        self.event = None

    def issue(self) -> None:
        """Enqueue the next chunk (a graph replay, or the eager remainder);
        with no steps left, the copy of the result to the host."""
        with torch.cuda.stream(self.stream):
            if self.left >= self.chunk:
                self.graph.replay()
                self.left -= self.chunk
            elif self.left > 0:
                self.shell.advance(self.state, self.left, self.time)
                self.left = 0
            else:
                self.host_out.copy_(self.state, non_blocking=True)
                self.host_time.copy_(self.time, non_blocking=True)
                self.left = -1
            self.event = torch.cuda.Event()
            self.event.record(self.stream)


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

    @property
    def time_to_solution(self) -> float:
        return self.t_done - self.t_arrival


class EnsembleServer:
    """Continuous-batching server over pooled slots (see module docstring)."""

    def __init__(self, hbm_budget: float, max_inflight: int = 8, chunk: int = 10, device: int | None = None):
        self.budget = hbm_budget
        self.max_inflight = max_inflight
        self.chunk = chunk
        self.device = torch.cuda.current_device() if device is None else device
        self.pool: dict[tuple, list[Slot]] = {}
        self.slot_bytes: dict[tuple, int] = {}
        self.in_use = 0.0

    @staticmethod
    def shape(req: Request) -> tuple[int, int, int]:
        return (req.nr, req.na, req.order)

    def warm(self, requests: list[Request], per_shape: int = 1) -> None:
        """Build slots ahead of time (contexts, buffers, graphs)."""
        for shp in sorted({self.shape(r) for r in requests}):
            for _ in range(per_shape - len(self.pool.get(shp, []))):
                s = Slot(shp, self.chunk, self.device)
                self.pool.setdefault(shp, []).append(s)
                self.slot_bytes[shp] = s.bytes

    def _acquire(self, req: Request) -> Slot | None:
        shp = self.shape(req)
        need = self.slot_bytes.get(shp, 0)
        if self.in_use + need > self.budget:
            return None
        idle = self.pool.setdefault(shp, [])
        slot = idle.pop() if idle else Slot(shp, self.chunk, self.device)
        self.slot_bytes[shp] = max(self.slot_bytes.get(shp, 0), slot.bytes)
        self.in_use += self.slot_bytes[shp]
        return slot

    def _release(self, slot: Slot) -> None:
        self.in_use -= self.slot_bytes[slot.shape]
        slot.req = None
        self.pool[slot.shape].append(slot)

    def run(self, requests: list[Request], states: dict[int, np.ndarray]) -> list[Result]:
        """Serve `requests` (arrival times relative to the call); `states`
        maps request id to its initial host state."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active: list[Slot] = []
        results: list[Result] = []
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_inflight:
                slot = self._acquire(pending[0])
                if slot is None:
                    break
                req = pending.pop(0)
                slot.start(req, states[req.rid], now)
                slot.issue()
                active.append(slot)
            progressed = False
            for slot in list(active):
                if slot.event is not None and not slot.event.query():
                    continue
                progressed = True
                if slot.left == -1:
                    req = slot.req
                    results.append(Result(req.rid, req.cells, req.steps, req.arrival, slot.t_start,
                                          time.perf_counter() - t0, slot.host_out.numpy().copy(),
                                          float(slot.host_time.item())))
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


def run_plain(requests: list[Request], states: dict[int, np.ndarray], device: int | None = None,
              shells: dict[tuple, Shell] | None = None) -> list[Result]:
    """The same requests one after another through eager per-solve launches
    (`Shell.advance`), with host copies in and out; contexts are cached by
    shape so neither path pays for context builds."""
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
        host = torch.from_numpy(states[req.rid]).pin_memory()
        ju = host.to(sh._dev, non_blocking=True)
        t = torch.zeros(1, dtype=torch.float64, device=sh._dev)
        sh.advance(ju, req.steps, t)
        out = ju.cpu().numpy()
        results.append(Result(req.rid, req.cells, req.steps, req.arrival, t_start, time.perf_counter() - t0, out,
                              float(t.item())))
    return results


def synthetic_requests(n: int, seed: int, rate_hz: float | None, steps: int,
                       radial=(32, 48, 64, 96), angular=(32, 48, 64), orders=(2, 4)) -> list[Request]:
    """Seeded requests: grid from `radial` x `angular`^2, scheme 50/50 from
    `orders`, cone speed U[500, 2000] km/s, half-width U[20, 60] deg,
    lat/lon U[-30, 30] deg, density ratio U[2, 6]; Poisson arrivals at
    `rate_hz` (all at t = 0 when None)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        if rate_hz:
            t += rng.exponential(1.0 / rate_hz)
        cone = Cone(speed_kms=rng.uniform(500, 2000), half_width_deg=rng.uniform(20, 60),
                    lat_deg=rng.uniform(-30, 30), lon_deg=rng.uniform(-30, 30), density_ratio=rng.uniform(2, 6))
        out.append(Request(rid, int(rng.choice(radial)), int(rng.choice(angular)), int(rng.choice(orders)), steps,
                           t if rate_hz else 0.0, cone))
    return out


def summarize(results: list[Result]) -> dict:
    tts = np.array([r.time_to_solution for r in results])
    span = max(r.t_done for r in results) - min(r.t_arrival for r in results)
    work = sum(r.cells * r.steps for r in results)
    return {"requests": len(results), "cell_updates": work, "makespan_s": span,
            "cell_updates_per_s": work / span, "p50_s": float(np.percentile(tts, 50)),
            "p99_s": float(np.percentile(tts, 99))}
