"""Host mirror of the reference's level/operator interface on one GPU.

`Shell` owns an hc_ctx (the level geometry the reference caches in
BoxOp_EulerCubedSphere::levelGeometry statics, src/BoxOp_EulerCubedSphere.H:
348-368) and exposes, over device tensors, the calls the reference's drivers
make:

    Shell.prepare      preStageLevel / prepareSecondOrderPrimitives
                       (src/BoxOp_PreStage.H:434-501)
    Shell.rhs          StageLevel (src/BoxOp_EulerCubedSphereImplem.H:961-1012)
    Shell.rk4_step     MBLevelRK::advance, order 4 (src/MHD_LevelRK.H:22-61)
    Shell.advance      the uniform driver's CFL + RK4 loop (exec/main.cpp:369-440)
    Shell.inv_dt_max   dtCFLSecondOrderHost (src/BoxOp_SecondOrderCFL.H:99-210)
    Shell.valid        validConservedState (src/BoxOp_EulerCubedSphereImplem.H:817-876)
    Shell.box_rhs      BoxOp_EulerCubedSphere::operator() on one box
    Shell.box_gravity  gravitySecondOrderPrimitives (src/BoxOp_Gravity.H:3-82)

All arithmetic runs in libhc_b200.so; torch supplies device memory and the
current CUDA stream only.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N

C_SR = 6.96e10          # cm, src/MHD_Constants.H:4
C_MP = 1.67262192e-24   # g, src/MHD_Constants.H:5


@dataclass
class Params:
    """Options of the second-order path (names follow src/Inputs_Parsing.H)."""
    nr: int = 32
    na: int = 32
    spatial_order: int = 2
    limiter: int = 3              # 0 unlimited, 1/2 minmod, 3 MC
    riemann_solver: int = 1       # 1 Rusanov, 2 Roe 8-wave
    divergence_cleaning: int = 1  # Powell
    sun_gravity: int = 0
    init_condition_type: int = 1  # analytic-wind inner boundary
    temporal_order: int = 4
    gamma: float = 5.0 / 3.0
    entropy_fix_coeff: float = 0.3
    cfl: float = 0.4
    inner_radius: float = 21.5 * C_SR
    outer_radius: float = 215.0 * C_SR
    radial_stretch: float = 1.5
    strength: float = 0.0
    spatial_operator: int = 2      # order 4: Berta WENOZ
    berta_detector_type: int = 0   # Jameson
    berta_fallback_type: int = 0   # 0 WENO3, 1 PLM
    berta_eta_d: float = 0.02
    autotune: int = 0              # order 2: time the stage tiles on the first step
    radial_offset: int = 0         # a radial slab: first radial cell within its shell
    radial_cells: int = 0          # radial cells of that shell (0: the level is the whole shell)

    def to_c(self) -> N.HcParams:
        p = N.HcParams()
        for k in ("nr", "na", "spatial_order", "limiter", "riemann_solver", "divergence_cleaning",
                  "sun_gravity", "init_condition_type", "temporal_order", "gamma", "entropy_fix_coeff",
                  "cfl", "inner_radius", "outer_radius", "radial_stretch", "strength", "spatial_operator",
                  "berta_detector_type", "berta_fallback_type", "berta_eta_d", "autotune", "radial_offset",
                  "radial_cells"):
            setattr(p, k, getattr(self, k))
        return p


@dataclass
class InitSpec:
    """Seeded synthetic initial state (kind 1): Parker-like wind with a
    Gaussian pressure pulse; see hc_init in include/hc_abi.h."""
    pulse_block: int = 0
    pulse_i: int = 0
    pulse_j: int = 0
    pulse_k: int = 0
    rho0: float = 700.0 * C_MP
    p0: float = 1.0e-7
    vr: float = 400.0e5
    b0: float = 5.0e-3
    r_ref: float = 21.5 * C_SR
    pulse_amp: float = 0.5
    pulse_width: float = 3.0

    def to_c(self) -> N.HcInit:
        s = N.HcInit()
        s.kind = 1
        for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref",
                  "pulse_amp", "pulse_width"):
            setattr(s, k, getattr(self, k))
        return s

    @staticmethod
    def seeded(seed: int, nr: int, na: int, margin: int = 6) -> "InitSpec":
        """Pulse centre at a seeded cell at least `margin` cells from every
        panel edge (and from the radial boundaries when the grid allows)."""
        rng = np.random.default_rng(seed)
        def pick(n):
            lo, hi = (margin, n - 1 - margin) if n - 1 - 2 * margin >= 0 else (0, n - 1)
            return int(rng.integers(lo, hi + 1))
        return InitSpec(pulse_block=int(rng.integers(0, 6)), pulse_i=pick(nr), pulse_j=pick(na), pulse_k=pick(na))


_PERM = ((1, 2, 0), (1, 2, 0), (1, 0, 2), (0, 1, 2), (1, 0, 2), (0, 1, 2))
_SIGN = ((1, -1, -1), (1, 1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1), (-1, -1, 1))


def cell_directions(na: int) -> np.ndarray:
    """Unit Cartesian direction of every cell centre, [6][3][k][j]
    (equiangular gnomonic panels, xi = (j + 1/2) / na)."""
    x = (np.arange(na) + 0.5) / na
    a = np.tan(-np.pi / 4 + np.pi / 2 * x)[None, :]
    c = np.tan(-np.pi / 4 + np.pi / 2 * x)[:, None]
    rho = np.sqrt(1 + a * a + c * c)
    q = (1 / rho, a / rho, c / rho)
    out = np.zeros((6, 3, na, na))
    for b in range(6):
        for k in range(3):
            out[b, k] = _SIGN[b][k] * np.broadcast_to(q[_PERM[b][k]], (na, na))
    return out


def perturbed_wind_state(params: Params, det: np.ndarray, dvolr: np.ndarray, seed: int, amp: float = 0.05,
                         spec: "InitSpec | None" = None) -> np.ndarray:
    """Synthetic level state JU [6][8][k][j][i] (host, float64): the
    Parker-like wind of InitSpec (rho ~ r^-2, v_r, p ~ r^-2 gamma,
    B_r ~ r^-2 sign(cos theta)) plus seeded tangential perturbations of
    relative size `amp` in v and B.  The tangential field is the surface
    curl of a seeded stream function times (r_ref / r)^2, so div B = 0 for
    the continuous field.  Cell averages are taken as J x point values at
    the cell centre (J = <det A> dVolr); det [6][k][j], dvolr [nr].  A
    radial slab (params.radial_cells > 0) gets its part of its shell's state."""
    spec = spec or InitSpec()
    nr, na, gam = params.nr, params.na, params.gamma
    rng = np.random.default_rng(seed)
    r0, r1, C = params.inner_radius, params.outer_radius, params.radial_stretch
    Rt = (r1 - r0) / np.expm1(C)
    r = r0 + Rt * np.expm1(C * (params.radial_offset + np.arange(nr) + 0.5) / (params.radial_cells or nr))
    s = spec.r_ref / r
    X = cell_directions(na)                                    # [6][3][k][j]

    def tangential_pattern(nmodes=4):
        """Surface gradient x rhat of psi = sum_m c_m sin(k_m . X + phi_m),
        normalised to unit max magnitude."""
        kv = rng.normal(size=(nmodes, 3)) * 2.0
        ph = rng.uniform(0, 2 * np.pi, nmodes)
        cm = rng.normal(size=nmodes)
        grad = np.zeros_like(X)
        for m in range(nmodes):
            arg = np.einsum("q,bqkj->bkj", kv[m], X) + ph[m]
            grad += cm[m] * np.cos(arg)[:, None] * kv[m][None, :, None, None]
        grad -= np.einsum("bqkj,bqkj->bkj", grad, X)[:, None] * X   # tangential part
        curl = np.cross(grad, X, axis=1)
        return curl / np.abs(curl).max()

    vt = tangential_pattern()
    bt = tangential_pattern()
    rho = spec.rho0 * s ** 2                                   # [nr]
    p = spec.p0 * s ** (2 * gam)
    sgn = np.sign(X[:, 2])                                     # sign(cos theta)
    Br = spec.b0 * s[None, None, None, :] ** 2 * sgn[..., None]
    ju = np.zeros((6, 8, na, na, nr))
    v = spec.vr * X[..., None] + amp * spec.vr * vt[..., None]                     # [6][3][k][j][i]
    B = Br[:, None] * X[..., None] + amp * spec.b0 * bt[..., None] * s[None, None, None, None, :] ** 2
    J = det[:, :, :, None] * dvolr[None, None, None, :]
    ju[:, 0] = rho * J
    ju[:, 1:4] = rho * v * J[:, None]
    ju[:, 5:8] = B * J[:, None]
    ju[:, 4] = (p / (gam - 1) + 0.5 * rho * (v ** 2).sum(1) + (B ** 2).sum(1) / (8 * np.pi)) * J
    return ju


def wind_box_state(params: Params, lo, hi, ghost: int, seed: int, spec: "InitSpec | None" = None) -> np.ndarray:
    """Native conserved averages of one box on valid.grow(ghost), [8][k][j][i]
    flattened: the Parker-like wind of InitSpec (rho ~ r^-2, v_r, p ~
    r^-2 gamma, B_r ~ r^-2) with seeded smooth tangential perturbations of a
    few percent (synthetic input for operator batches; the native basis
    has the radial unit vector as its first column)."""
    spec = spec or InitSpec()
    rng = np.random.default_rng(seed)
    gam = params.gamma
    r0, r1, C = params.inner_radius, params.outer_radius, params.radial_stretch
    Rt = (r1 - r0) / np.expm1(C)
    i = np.arange(lo[0] - ghost, hi[0] + ghost + 1)
    j = np.arange(lo[1] - ghost, hi[1] + ghost + 1)
    k = np.arange(lo[2] - ghost, hi[2] + ghost + 1)
    r = r0 + Rt * np.expm1(C * (i + 0.5) / params.nr)
    s = spec.r_ref / r
    ph = rng.uniform(0, 2 * np.pi, 3)
    h = 1.0 / params.na
    ang = (np.sin(2 * np.pi * (j + 0.5) * h + ph[0])[None, :, None]
           * np.cos(2 * np.pi * (k + 0.5) * h + ph[1])[:, None, None])
    rho = spec.rho0 * s ** 2 * (1 + 0.05 * ang)
    p = spec.p0 * s ** (2 * gam) * (1 + 0.02 * ang)
    U = np.zeros((8,) + rho.shape)
    U[0] = rho
    U[1] = rho * spec.vr
    U[2] = rho * spec.vr * 0.01 * ang
    U[3] = rho * spec.vr * 0.01 * np.cos(2 * np.pi * (j + 0.5) * h + ph[2])[None, :, None]
    U[5] = spec.b0 * s ** 2
    U[6] = 0.02 * spec.b0 * s * ang
    U[4] = p / (gam - 1) + 0.5 * rho * spec.vr ** 2 + U[5] ** 2 / (8 * np.pi)
    return np.ascontiguousarray(U.reshape(-1))


@dataclass
class ConeSpec:
    """Fitted parameters of a finite cone-CME cloud (hc_cone_spec; the
    reference's CMEParameters of field model 4 with an analytic cone)."""
    lat_deg: float = 0.0
    lon_deg: float = 0.0
    half_angle_deg: float = 30.0
    apex_speed: float = 1200.0          # km/s at reference_time
    wind_speed: float = 400.0           # km/s (drag-based model)
    drag_gamma: float = 0.0             # 1/km (0: ballistic)
    reference_height: float = 21.5      # leading edge at reference_time, solar radii
    reference_time: float = 0.0         # s
    density: float = 4 * 700.0 * C_MP   # g/cm^3
    temperature: float = 1.0e6          # K

    def to_c(self) -> N.HcConeSpec:
        s = N.HcConeSpec()
        for k in N._CONE_SPEC:
            setattr(s, k, getattr(self, k))
        return s

    @classmethod
    def on_inner_boundary(cls, inner_radius: float, **kw) -> "ConeSpec":
        """A cloud that lies wholly inside the shell at reference_time,
        touching the inner boundary: leading edge at r_inner (1 + 2 sin a)."""
        spec = cls(**kw)
        a = np.sin(np.radians(spec.half_angle_deg))
        spec.reference_height = inner_radius * (1.0 + 2.0 * a) / C_SR
        return spec


def o4_variants() -> np.ndarray:
    """Minimum resident CTAs per SM of each register-cap variant of the
    fourth-order operator's tuned kernels, [kernel][variant]: reconstruction,
    Roe point dissipation, fused face chain (hc_o4_variants)."""
    lib = N.lib()
    n = lib.hc_o4_variants(None, 0)
    out = (C.c_int * (3 * n))()
    lib.hc_o4_variants(out, 3 * n)
    return np.array(out[:], dtype=np.int64).reshape(3, n)


def stage_tiles() -> np.ndarray:
    """Candidate tiles of the order-2 stage kernel, [tiles][5]: cells x, y,
    z, min CTAs per SM with Rusanov, with Roe (hc_stage_tiles)."""
    lib = N.lib()
    n = lib.hc_stage_tiles(None, 0)
    out = (C.c_int * (5 * n))()
    lib.hc_stage_tiles(out, n)
    return np.array(out[:], dtype=np.int64).reshape(n, 5)


def prepare_cone(spec: ConeSpec, inner_radius: float) -> N.HcCone:
    """hc_cone_prepare: the cloud's geometry and timing (host arithmetic)."""
    out = N.HcCone()
    s = spec.to_c()
    N.check(N.lib().hc_cone_prepare(C.byref(s), inner_radius, C.byref(out)), "hc_cone_prepare")
    return out


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("expected a contiguous float64 CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class _DeviceArray:
    """A float64 device buffer owned by the library, for a torch view."""

    def __init__(self, ptr: int, shape: tuple[int, ...]):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


class Shell:
    """One cubed-sphere level (six panels, one box each) on one GPU."""

    def __init__(self, params: Params, device: int | None = None):
        if not torch.cuda.is_available():
            raise N.HcError("heliocubed_b200 needs a CUDA device; there is no CPU path")
        self.params = params
        self.device = torch.cuda.current_device() if device is None else device
        self._lib = N.lib()
        self._ctx = C.c_void_p()
        self._cp = params.to_c()
        with torch.cuda.device(self.device):
            N.check(self._lib.hc_ctx_create(C.byref(self._cp), self.device, C.byref(self._ctx)), "hc_ctx_create")
        self.nv = int(self._lib.hc_level_state_size(self._ctx))
        self.ng = int(self._lib.hc_level_primitive_size(self._ctx))
        self._scalar = torch.zeros(4, dtype=torch.float64, device=self._dev)
        self._flag = torch.zeros(1, dtype=torch.int32, device=self._dev)

    @property
    def _dev(self) -> torch.device:
        return torch.device("cuda", self.device)

    @property
    def cells(self) -> int:
        return 6 * self.params.nr * self.params.na ** 2

    def close(self) -> None:
        if self._ctx:
            self._lib.hc_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- storage ---------------------------------------------------------
    def new_state(self) -> torch.Tensor:
        return torch.zeros(self.nv, dtype=torch.float64, device=self._dev)

    def new_primitive(self) -> torch.Tensor:
        return torch.zeros(self.ng, dtype=torch.float64, device=self._dev)

    def state_view(self, ju: torch.Tensor) -> torch.Tensor:
        """[panel][component][k][j][i] view of a level state."""
        p = self.params
        return ju.view(6, 8, p.na, p.na, p.nr)

    # -- level operations ------------------------------------------------
    def init(self, spec: InitSpec, ju: torch.Tensor | None = None) -> torch.Tensor:
        ju = self.new_state() if ju is None else ju
        s = spec.to_c()
        N.check(self._lib.hc_level_init(self._ctx, C.byref(s), _ptr(ju), _stream()), "hc_level_init")
        return ju

    def init_perturbed_wind(self, seed: int, amp: float = 0.05) -> torch.Tensor:
        """Level state of perturbed_wind_state (built on the host, copied)."""
        p = self.params
        det = self.geometry(4).reshape(6, p.na, p.na)
        dvolr = self.geometry(0).reshape(p.nr + 1, 4)[:p.nr, 3]
        ju = perturbed_wind_state(p, det, dvolr, seed, amp)
        return torch.from_numpy(np.ascontiguousarray(ju.reshape(-1))).to(self._dev)

    def set_cme_schedule(self, events) -> None:
        """hc_level_set_cme_schedule on the current stream: events are
        hc_cme_event structures or prepared cones (their schedule events via
        hc_cone_event)."""
        n = len(events)
        arr = (N.HcCmeEvent * max(n, 1))()
        for i, e in enumerate(events):
            if isinstance(e, N.HcCone):
                N.check(self._lib.hc_cone_event(C.byref(e), C.byref(arr[i])), "hc_cone_event")
            else:
                arr[i] = e
        N.check(self._lib.hc_level_set_cme_schedule(self._ctx, arr, n, _stream()), "hc_level_set_cme_schedule")

    def set_inlet(self, cones) -> None:
        """hc_level_set_inlet: prepared cones fed through the inner boundary
        while they cross it (order 2)."""
        n = len(cones)
        arr = (N.HcCone * max(n, 1))(*cones)
        N.check(self._lib.hc_level_set_inlet(self._ctx, arr, n, _stream()), "hc_level_set_inlet")

    def autotune(self, ju: torch.Tensor) -> tuple[tuple[int, ...], np.ndarray]:
        """hc_ctx_autotune with the state `ju` (not modified).  Order 2:
        ((RK stage tile, operator tile), median ms [2][tiles]).  Order 4:
        ((reconstruction, Roe point, face chain variant), operator ms
        [3][variants])."""
        if self.params.spatial_order == 4:
            rows, n = 3, o4_variants().shape[1]
        else:
            rows, n = 2, stage_tiles().shape[0]
        tiles = (C.c_int * rows)()
        ms = np.zeros(rows * n)
        N.check(self._lib.hc_ctx_autotune(self._ctx, _ptr(ju), tiles, ms.ctypes.data_as(C.c_void_p), _stream()),
                "hc_ctx_autotune")
        return tuple(tiles[:]), ms.reshape(rows, n)

    def set_o4_variants(self, recon: int = -1, roe: int = -1, final: int = -1) -> None:
        v = (C.c_int * 3)(recon, roe, final)
        N.check(self._lib.hc_ctx_set_o4_variants(self._ctx, v), "hc_ctx_set_o4_variants")

    def set_tiles(self, tile_rk: int = -1, tile_rhs: int = -1) -> None:
        N.check(self._lib.hc_ctx_set_tiles(self._ctx, tile_rk, tile_rhs), "hc_ctx_set_tiles")

    def insert_cone(self, cone: N.HcCone, time: float, ju: torch.Tensor, stats: bool = False) -> torch.Tensor | None:
        """Volume insertion of a prepared cone cloud into `ju` at `time`
        (hc_level_insert_cone); with `stats` a device tensor [cells, grams]."""
        out = torch.zeros(2, dtype=torch.float64, device=self._dev) if stats else None
        N.check(self._lib.hc_level_insert_cone(self._ctx, C.byref(cone), time, _ptr(ju), _ptr(out), _stream()),
                "hc_level_insert_cone")
        return out

    def prepare(self, ju: torch.Tensor, t: float = 0.0, w: torch.Tensor | None = None) -> torch.Tensor:
        w = self.new_primitive() if w is None else w
        N.check(self._lib.hc_level_prepare(self._ctx, _ptr(ju), _ptr(w), t, _stream()), "hc_level_prepare")
        return w

    def rhs(self, w: torch.Tensor, k: torch.Tensor | None = None) -> torch.Tensor:
        k = self.new_state() if k is None else k
        N.check(self._lib.hc_level_rhs(self._ctx, _ptr(w), _ptr(k), _stream()), "hc_level_rhs")
        return k

    def prepare_cartesian(self, ju: torch.Tensor, t: float = 0.0, w: torch.Tensor | None = None,
                          cart: torch.Tensor | None = None) -> tuple[torch.Tensor, torch.Tensor]:
        """Fourth order: hc_level_prepare keeping the Cartesian averages
        (hc_level_prepare_cartesian); returns (w, cart)."""
        w = self.new_primitive() if w is None else w
        if cart is None:
            cart = torch.empty(int(self._lib.hc_level_cartesian_size(self._ctx)), dtype=torch.float64,
                               device=self._dev)
        N.check(self._lib.hc_level_prepare_cartesian(self._ctx, _ptr(ju), _ptr(w), _ptr(cart), t, _stream()),
                "hc_level_prepare_cartesian")
        return w, cart

    def rhs_fluxes(self, w: torch.Tensor, k: torch.Tensor, fluxes=None) -> None:
        """Fourth order: the AMR level evaluation (hc_level_rhs_fluxes): k
        with the panel seams reconciled, fluxes[d] each panel's face fluxes."""
        arr = (C.c_void_p * 3)(*[_ptr(f) if f is not None else None for f in fluxes]) if fluxes is not None else None
        N.check(self._lib.hc_level_rhs_fluxes(self._ctx, _ptr(w), _ptr(k), arr, _stream()), "hc_level_rhs_fluxes")

    def rk4_step(self, ju: torch.Tensor, dt: float, t: float = 0.0) -> None:
        N.check(self._lib.hc_level_rk4_step(self._ctx, _ptr(ju), dt, t, _stream()), "hc_level_rk4_step")

    def rk4_stage(self, ju: torch.Tensor, stage: int, dt: float = 0.0, t: float = 0.0,
                  inv_dt: torch.Tensor | None = None, time: torch.Tensor | None = None) -> None:
        """Stage `stage` of rk4_step (stages 0..3 in order make one step);
        with inv_dt (device) dt = cfl / inv_dt, with time (device) the stage
        time is t + time + c_s dt."""
        N.check(self._lib.hc_level_rk4_stage(self._ctx, _ptr(ju), stage, dt, t, _ptr(inv_dt), _ptr(time),
                                             _stream()), "hc_level_rk4_stage")

    def set_radial_window(self, lo: int, hi: int) -> None:
        """Order 4: the RK4 stages evaluate the operator on radial cells
        [lo, hi) only (0, 0: every cell); the others get rhs 0."""
        N.check(self._lib.hc_level_set_radial_window(self._ctx, lo, hi), "hc_level_set_radial_window")

    def stage_state(self, ju: torch.Tensor, stage: int) -> tuple[torch.Tensor, int]:
        """The buffer stage `stage` reads, as a (rows, radial) view sharing
        its memory, and the column of the level's first radial cell."""
        data, rows, n, first = C.c_void_p(), C.c_long(), C.c_int(), C.c_int()
        N.check(self._lib.hc_level_stage_state(self._ctx, _ptr(ju), stage, C.byref(data), C.byref(rows), C.byref(n),
                                               C.byref(first)), "hc_level_stage_state")
        if data.value == ju.data_ptr():
            return ju.view(rows.value, n.value), first.value
        return torch.as_tensor(_DeviceArray(data.value, (rows.value, n.value)), device=self._dev), first.value

    def advance(self, ju: torch.Tensor, nsteps: int, time: torch.Tensor | None = None,
                dt_out: torch.Tensor | None = None) -> None:
        """nsteps RK4 steps with dt = cfl / max CFL rate, computed on device."""
        N.check(self._lib.hc_level_advance_cfl(self._ctx, _ptr(ju), nsteps, _ptr(time), _ptr(dt_out), _stream()),
                "hc_level_advance_cfl")

    def capture_advance(self, ju: torch.Tensor, nsteps: int, time: torch.Tensor,
                        dt_out: torch.Tensor | None = None) -> "torch.cuda.CUDAGraph":
        """Capture `advance(ju, nsteps, time)` into a CUDA graph (the launch
        sequence has no host synchronisation or allocation).  One eager run
        on a side stream precedes the capture, so ju advances by nsteps."""
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=self._dev)
        side.wait_stream(torch.cuda.current_stream(self._dev))
        with torch.cuda.stream(side):
            self.advance(ju, nsteps, time, dt_out)
        torch.cuda.current_stream(self._dev).wait_stream(side)
        with torch.cuda.graph(g):
            self.advance(ju, nsteps, time, dt_out)
        return g

    def inv_dt_max(self, ju: torch.Tensor) -> torch.Tensor:
        out = torch.zeros(1, dtype=torch.float64, device=self._dev)
        N.check(self._lib.hc_level_dt_cfl(self._ctx, _ptr(ju), _ptr(out), _stream()), "hc_level_dt_cfl")
        return out

    def valid(self, ju: torch.Tensor) -> bool:
        N.check(self._lib.hc_level_valid(self._ctx, _ptr(ju), C.c_void_p(self._flag.data_ptr()), _stream()),
                "hc_level_valid")
        return bool(self._flag.item())

    def box_rhs(self, box: N.HcBox, w: torch.Tensor, rhs: torch.Tensor, fluxes=None, panel=None,
                scale: float = 1.0) -> None:
        fl = (C.c_void_p * 3)(*[(f.data_ptr() if f is not None else None) for f in fluxes]) if fluxes else None
        pn = (C.c_void_p * 6)(*[(f.data_ptr() if f is not None else None) for f in panel]) if panel else None
        N.check(self._lib.hc_box_rhs(self._ctx, C.byref(box), _ptr(w), pn, scale, _ptr(rhs), fl, _stream()),
                "hc_box_rhs")

    def box_rhs_o4(self, box: N.HcBox, usph: torch.Tensor, rhs: torch.Tensor, fluxes=None,
                   scale: float = 1.0) -> None:
        """Fourth-order Berta operator on one box (BertaOperator):
        usph are native conserved averages on valid.grow(ghost >= 5)."""
        fl = (C.c_void_p * 3)(*[(f.data_ptr() if f is not None else None) for f in fluxes]) if fluxes else None
        N.check(self._lib.hc_box_rhs_o4(self._ctx, C.byref(box), _ptr(usph), scale, _ptr(rhs), fl, _stream()),
                "hc_box_rhs_o4")

    def box_gravity(self, box: N.HcBox, w: torch.Tensor, rhs: torch.Tensor) -> None:
        N.check(self._lib.hc_box_gravity(self._ctx, C.byref(box), _ptr(w), _ptr(rhs), _stream()), "hc_box_gravity")

    def o4_batch(self, works, scale: float = 1.0) -> "O4Batch":
        """A batch of boxes of any sizes for the fourth-order operator:
        works = [(box, usph, rhs, fluxes or None), ...] over device tensors."""
        return O4Batch(self, works, scale)

    def box_gravity_o4(self, box: N.HcBox, usph: torch.Tensor, rhs: torch.Tensor) -> None:
        """Gravity_Euler (src/BoxOp_Gravity.H:84-164) on one box of native
        averages (valid.grow(ghost >= 1)); rhs[valid] += source."""
        N.check(self._lib.hc_box_gravity_o4(self._ctx, C.byref(box), _ptr(usph), _ptr(rhs), _stream()),
                "hc_box_gravity_o4")

    def geometry(self, what: int) -> np.ndarray:
        n = self._lib.hc_geometry_export(self._ctx, what, None)
        if n < 0:
            raise N.HcError(f"unknown geometry table {what}")
        out = np.zeros(n)
        self._lib.hc_geometry_export(self._ctx, what, C.c_void_p(out.ctypes.data))
        return out


def make_box(lo, hi, ghost: int, block: int) -> N.HcBox:
    b = N.HcBox()
    for d in range(3):
        b.lo[d] = lo[d]
        b.hi[d] = hi[d]
    b.ghost = ghost
    b.block = block
    return b


class O4Batch:
    """hc_o4_batch: the fourth-order operator on many boxes of any sizes, each
    operator kernel one launch over all of them.  Keeps the tensors alive."""

    def __init__(self, shell: Shell, works, scale: float = 1.0):
        self.shell = shell
        self._keep = []
        arr = (N.HcBoxWork * len(works))()
        for q, (box, usph, rhs, fluxes) in enumerate(works):
            arr[q].box = box
            arr[q].usph = usph.data_ptr()
            arr[q].rhs = rhs.data_ptr()
            for d in range(3):
                arr[q].flux[d] = fluxes[d].data_ptr() if fluxes is not None and fluxes[d] is not None else None
            self._keep.append((usph, rhs, fluxes))
        h = C.c_void_p()
        N.check(shell._lib.hc_o4_batch_create(shell._ctx, arr, len(works), scale, C.byref(h)), "hc_o4_batch_create")
        self._h = h

    def rhs(self) -> None:
        N.check(self.shell._lib.hc_o4_batch_rhs(self.shell._ctx, self._h, _stream()), "hc_o4_batch_rhs")

    def close(self) -> None:
        if self._h:
            self.shell._lib.hc_o4_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """hc_ensemble: fourth-order levels of any sizes advanced together, each
    with its own state, CFL dt, model time and insertion schedule, the stage
    operator of all of them one batched launch per kernel.  The shells must
    outlive the ensemble and must not step on their own while it is used."""

    def __init__(self, shells: list[Shell]):
        if not shells:
            raise ValueError("an ensemble needs at least one level")
        self.shells = list(shells)
        self._lib = shells[0]._lib
        arr = (C.c_void_p * len(shells))(*[s._ctx.value for s in shells])
        h = C.c_void_p()
        N.check(self._lib.hc_ensemble_create(arr, len(shells), C.byref(h)), "hc_ensemble_create")
        self._h = h

    def advance(self, states: list[torch.Tensor], nsteps: int, times: list[torch.Tensor] | None = None,
                dts: list[torch.Tensor] | None = None) -> None:
        """nsteps CFL steps of every level (states[q] of shells[q]; times[q]
        and dts[q] device doubles as in Shell.advance)."""
        m = len(self.shells)
        if len(states) != m or (times is not None and len(times) != m) or (dts is not None and len(dts) != m):
            raise ValueError("one state (and time, dt) per level")

        def ptrs(ts):
            return (C.c_void_p * m)(*[_ptr(t) for t in ts]) if ts is not None else None

        N.check(self._lib.hc_ensemble_advance_cfl(self._h, ptrs(states), nsteps, ptrs(times), ptrs(dts), _stream()),
                "hc_ensemble_advance_cfl")

    def close(self) -> None:
        if self._h:
            self._lib.hc_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def amr_exchange_copies(boxes, ghost: int):
    """Same-panel ghost exchange of one level as region copies
    (hc_copy_box descriptors without the array pointers): for every ordered
    pair of boxes (b, a) on the same panel, the cells of box a's storage
    region (valid.grow(ghost)) that lie in box b's valid region are copied
    from b to a with the identity index map.  boxes: (panel, lo, hi) per
    box, inclusive valid bounds.  Returns dicts with src_box and dst_box (box
    indices), lo, hi, perm, sign and shift; the caller adds the arrays and
    their boxes (valid.grow(ghost)) and passes them to AmrPlan.set_copies.
    Copies across panels (signed permutations of the index space) are the
    caller's."""
    out = []
    for a, (pa, alo, ahi) in enumerate(boxes):
        slo = [alo[d] - ghost for d in range(3)]
        shi = [ahi[d] + ghost for d in range(3)]
        for b, (pb, blo, bhi) in enumerate(boxes):
            if b == a or pb != pa:
                continue
            lo = [max(slo[d], blo[d]) for d in range(3)]
            hi = [min(shi[d], bhi[d]) for d in range(3)]
            if any(lo[d] > hi[d] for d in range(3)):
                continue
            out.append({"src_box": b, "dst_box": a, "lo": lo, "hi": hi, "perm": (0, 1, 2), "sign": (1, 1, 1),
                        "shift": (0, 0, 0)})
    return out


def amr_cf_weights(ratio: int, child: int) -> np.ndarray:
    """hc_amr_cf_weights: the five coarse weights of child `child` of a cell
    refined by `ratio` (host arithmetic; no device needed)."""
    w = (C.c_double * 5)()
    N.check(N.lib().hc_amr_cf_weights(ratio, child, w), "hc_amr_cf_weights")
    return np.array(w[:])


class AmrPlan:
    """The AMR Runge-Kutta stage logic of a set of boxes (any levels, any
    sizes): hc_amr_plan_create / hc_amr_rk_stage / hc_amr_restrict.

    boxes: (state, stage, [rk0, rk1, rk2, rk3]) device tensors of 8 x
    ncells doubles each.  restricts: dicts with fine, coarse (device
    tensors), fine_lo, fine_n, coarse_lo, coarse_n, lo, hi, ratio (3 ints
    each).  The tensors must outlive the plan."""

    def __init__(self, shell: "Shell", boxes, restricts=()):
        self._shell = shell
        self._lib = shell._lib
        nb, nr = len(boxes), len(restricts)
        bx = (N.HcRkBox * max(nb, 1))()
        for b, (state, stage, rk) in enumerate(boxes):
            bx[b].ncells = state.numel() // 8
            bx[b].state = state.data_ptr()
            bx[b].stage = stage.data_ptr()
            for q in range(4):
                bx[b].rk[q] = rk[q].data_ptr()
        rx = (N.HcRestrictBox * max(nr, 1))()
        for r, d in enumerate(restricts):
            rx[r].fine = d["fine"].data_ptr()
            rx[r].coarse = d["coarse"].data_ptr()
            for k in ("fine_lo", "fine_n", "coarse_lo", "coarse_n", "lo", "hi", "ratio"):
                getattr(rx[r], k)[:] = list(d[k])
        self._h = C.c_void_p()
        N.check(self._lib.hc_amr_plan_create(shell._ctx, bx, nb, rx, nr, C.byref(self._h)), "hc_amr_plan_create")

    def rk_stage(self, order: int, stage: int, dt: float) -> None:
        N.check(self._lib.hc_amr_rk_stage(self._shell._ctx, self._h, order, stage, dt, _stream()), "hc_amr_rk_stage")

    def restrict(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_restrict(self._shell._ctx, self._h, first, count, _stream()), "hc_amr_restrict")

    def set_reflux(self, patches) -> None:
        """patches: dicts with fine_flux, coarse_flux, rhs (device tensors),
        fine_lo, fine_n, coarse_lo, coarse_n, rhs_lo, rhs_n, lo, hi, ratio
        (3 ints each), dir, fine_side and scale (hc_reflux_box)."""
        n = len(patches)
        arr = (N.HcRefluxBox * max(n, 1))()
        for r, d in enumerate(patches):
            arr[r].fine_flux = d["fine_flux"].data_ptr()
            arr[r].coarse_flux = d["coarse_flux"].data_ptr()
            arr[r].rhs = d["rhs"].data_ptr()
            for k in ("fine_lo", "fine_n", "coarse_lo", "coarse_n", "rhs_lo", "rhs_n", "lo", "hi", "ratio"):
                getattr(arr[r], k)[:] = list(d[k])
            arr[r].dir, arr[r].fine_side, arr[r].scale = d["dir"], d["fine_side"], d["scale"]
        N.check(self._lib.hc_amr_plan_set_reflux(self._h, arr, n), "hc_amr_plan_set_reflux")

    def reflux(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_reflux(self._shell._ctx, self._h, first, count, _stream()), "hc_amr_reflux")

    def set_cf_interp(self, boxes) -> None:
        """boxes: dicts with coarse, fine (device tensors of ncomp x box
        cells), coarse_lo, coarse_n, fine_lo, fine_n, valid_lo, valid_hi,
        ratio (3 ints each) and ncomp (hc_cf_box)."""
        n = len(boxes)
        arr = (N.HcCfBox * max(n, 1))()
        for b, d in enumerate(boxes):
            arr[b].coarse = d["coarse"].data_ptr()
            arr[b].fine = d["fine"].data_ptr()
            for k in ("coarse_lo", "coarse_n", "fine_lo", "fine_n", "valid_lo", "valid_hi", "ratio"):
                getattr(arr[b], k)[:] = list(d[k])
            arr[b].ncomp = d["ncomp"]
        N.check(self._lib.hc_amr_plan_set_cf_interp(self._h, arr, n), "hc_amr_plan_set_cf_interp")

    def cf_interpolate(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_cf_interpolate(self._shell._ctx, self._h, first, count, _stream()),
                "hc_amr_cf_interpolate")

    def set_copies(self, copies) -> None:
        """copies: dicts with src, dst (device tensors), src_lo, src_n,
        dst_lo, dst_n, lo, hi, perm, sign, shift (3 ints each) and ncomp
        (hc_copy_box)."""
        n = len(copies)
        arr = (N.HcCopyBox * max(n, 1))()
        for q, d in enumerate(copies):
            arr[q].src = d["src"].data_ptr()
            arr[q].dst = d["dst"].data_ptr()
            for k in ("src_lo", "src_n", "dst_lo", "dst_n", "lo", "hi", "perm", "sign", "shift"):
                getattr(arr[q], k)[:] = list(d[k])
            arr[q].ncomp = d["ncomp"]
        N.check(self._lib.hc_amr_plan_set_copies(self._h, arr, n), "hc_amr_plan_set_copies")

    def copy(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_copy(self._shell._ctx, self._h, first, count, _stream()), "hc_amr_copy")

    def set_cf_fine(self, boxes) -> None:
        """boxes: dicts with jac, donor, state, mapped, out (device tensors)
        and their *_lo / *_n boxes, valid_lo, valid_hi, block_lo, block_hi
        (3 ints each) (hc_cf_fine_box)."""
        n = len(boxes)
        arr = (N.HcCfFineBox * max(n, 1))()
        for b, d in enumerate(boxes):
            for a in ("jac", "donor", "state", "mapped", "out"):
                setattr(arr[b], a, d[a].data_ptr())
                getattr(arr[b], a + "_lo")[:] = list(d[a + "_lo"])
                getattr(arr[b], a + "_n")[:] = list(d[a + "_n"])
            for k in ("valid_lo", "valid_hi", "block_lo", "block_hi"):
                getattr(arr[b], k)[:] = list(d[k])
        N.check(self._lib.hc_amr_plan_set_cf_fine(self._h, arr, n), "hc_amr_plan_set_cf_fine")

    def cf_mapped(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_cf_mapped(self._shell._ctx, self._h, first, count, _stream()), "hc_amr_cf_mapped")

    def cf_quotient(self, first: int, count: int) -> None:
        N.check(self._lib.hc_amr_cf_quotient(self._shell._ctx, self._h, first, count, _stream()),
                "hc_amr_cf_quotient")

    def set_native(self, boxes) -> None:
        """boxes: dicts with cart and usph (device tensors), cart_lo, cart_n,
        usph_lo, usph_n (3 ints each) and block (hc_native_box)."""
        n = len(boxes)
        arr = (N.HcNativeBox * max(n, 1))()
        for b, d in enumerate(boxes):
            arr[b].cart = d["cart"].data_ptr()
            arr[b].usph = d["usph"].data_ptr()
            for k in ("cart_lo", "cart_n", "usph_lo", "usph_n"):
                getattr(arr[b], k)[:] = list(d[k])
            arr[b].block = d["block"]
        N.check(self._lib.hc_amr_plan_set_native(self._h, arr, n), "hc_amr_plan_set_native")

    def native(self, first: int, count: int, t: float) -> None:
        """Native averages and radial ghosts of boxes first .. first+count-1
        at time t, with the geometry of this plan's shell (hc_amr_native)."""
        N.check(self._lib.hc_amr_native(self._shell._ctx, self._h, first, count, t, _stream()), "hc_amr_native")

    def close(self) -> None:
        if self._h:
            self._lib.hc_amr_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

