"""ctypes bindings of the oracle (libhc_oracle.so) and of the reference pin
(_ref/libhcref.so).  Test infrastructure only: used by tests/, by
__graft_entry__.smoke() as the checker and by bench.py's CPU-baseline arm.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_I = C.POINTER(C.c_int)


class HcParams(C.Structure):
    """Mirror of hc_params in include/hc_abi.h."""
    _fields_ = [
        ("spatial_order", C.c_int), ("limiter", C.c_int), ("riemann_solver", C.c_int),
        ("divergence_cleaning", C.c_int), ("sun_gravity", C.c_int),
        ("init_condition_type", C.c_int), ("temporal_order", C.c_int),
        ("nr", C.c_int), ("na", C.c_int), ("spatial_operator", C.c_int), ("berta_detector_type", C.c_int),
        ("berta_fallback_type", C.c_int), ("autotune", C.c_int),
        ("radial_offset", C.c_int), ("radial_cells", C.c_int), ("reserved_i", C.c_int * 1),
        ("gamma", C.c_double), ("entropy_fix_coeff", C.c_double), ("cfl", C.c_double),
        ("inner_radius", C.c_double), ("outer_radius", C.c_double),
        ("radial_stretch", C.c_double), ("strength", C.c_double), ("berta_eta_d", C.c_double),
        ("reserved_d", C.c_double * 6),
    ]


class HcBox(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("ghost", C.c_int), ("block", C.c_int)]


class HcInit(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("pulse_block", C.c_int), ("pulse_i", C.c_int), ("pulse_j", C.c_int),
        ("pulse_k", C.c_int), ("reserved_i", C.c_int * 3),
        ("rho0", C.c_double), ("p0", C.c_double), ("vr", C.c_double), ("b0", C.c_double),
        ("r_ref", C.c_double), ("pulse_amp", C.c_double), ("pulse_width", C.c_double),
        ("reserved_d", C.c_double * 4),
    ]


CONE_SPEC_FIELDS = ("lat_deg", "lon_deg", "half_angle_deg", "apex_speed", "wind_speed", "drag_gamma",
                    "reference_height", "reference_time", "density", "temperature")
CONE_FIELDS = ("radius", "entry_shift", "entry_time", "speed", "end_time", "insertion_time", "density",
               "temperature")


class HcConeSpec(C.Structure):
    """Mirror of hc_cone_spec in include/hc_abi.h."""
    _fields_ = [(n, C.c_double) for n in CONE_SPEC_FIELDS] + [("reserved", C.c_double * 6)]


class HcCmeEvent(C.Structure):
    """Mirror of hc_cme_event in include/hc_abi.h."""
    _fields_ = [("insertion_time", C.c_double), ("feeding_end", C.c_double), ("boundary", C.c_int),
                ("reserved", C.c_int)]


class HcCone(C.Structure):
    """Mirror of hc_cone in include/hc_abi.h."""
    _fields_ = [("axis", C.c_double * 3)] + [(n, C.c_double) for n in CONE_FIELDS] + [("reserved", C.c_double * 6)]


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run python oracle/build.py")
    return C.CDLL(path)


_orc = None
_ref = None


_lib_path = None


def use_library(path: str) -> None:
    """Load the oracle from `path` (a build of the same source, e.g. the
    -march=native copy of the timed CPU baseline) instead of the shipped
    library; only before the first call of lib()."""
    global _lib_path
    if _orc is not None and path != _lib_path:
        raise RuntimeError("the oracle library is already loaded")
    _lib_path = path


def lib() -> C.CDLL:
    global _orc
    if _orc is None:
        L = _load(_lib_path or os.path.join(HERE, "libhc_oracle.so"))
        L.orc_level_create.restype = C.c_void_p
        L.orc_level_create.argtypes = [C.POINTER(HcParams)]
        L.orc_level_destroy.argtypes = [C.c_void_p]
        L.orc_box_rhs.argtypes = [C.c_void_p, C.POINTER(HcBox), _D, C.POINTER(_D), C.c_double, _D, C.POINTER(_D)]
        L.orc_box_gravity.argtypes = [C.c_void_p, C.POINTER(HcBox), _D, _D]
        L.orc_box_gravity_o4.argtypes = [C.c_void_p, C.POINTER(HcBox), _D, _D]
        L.orc_box_rhs_o4.argtypes = [C.c_void_p, C.POINTER(HcBox), _D, C.c_double, _D, C.POINTER(_D)]
        L.orc_level_prepare.argtypes = [C.c_void_p, _D, _D, C.c_double]
        L.orc_level_rhs.argtypes = [C.c_void_p, _D, _D]
        L.orc_level_rk4_step.argtypes = [C.c_void_p, _D, C.c_double, C.c_double]
        L.orc_level_inv_dt.restype = C.c_double
        L.orc_level_inv_dt.argtypes = [C.c_void_p, _D]
        L.orc_level_valid.argtypes = [C.c_void_p, _D]
        L.orc_level_init.argtypes = [C.c_void_p, C.POINTER(HcInit), _D]
        L.orc_geometry.restype = C.c_long
        L.orc_geometry.argtypes = [C.c_void_p, C.c_int, _D]
        L.orc_roe8.argtypes = [_D, _D, C.c_double, C.c_double, C.c_int, _D]
        L.orc_rusanov.argtypes = [_D, _D, C.c_double, _D]
        L.orc_frame.argtypes = [_D, _D, _D]
        L.orc_face_flux.argtypes = [_D, _D, _D, C.c_double, C.c_double, C.c_double, C.c_int, _D]
        L.orc_plm.argtypes = [_D, _D, _D, _D, C.c_int, _D, _D]
        L.orc_cart_prim.argtypes = [_D, C.c_double, C.c_double, _D]
        L.orc_cone_prepare.argtypes = [C.POINTER(HcConeSpec), C.c_double, C.POINTER(HcCone)]
        L.orc_cone_cell.argtypes = [C.POINTER(HcCone), C.c_double, _D, _D, C.c_double, _D]
        L.orc_level_insert_cone.argtypes = [C.c_void_p, C.POINTER(HcCone), C.c_double, _D, _D]
        L.orc_cme_schedule.argtypes = [C.POINTER(HcCmeEvent), C.c_int, C.c_double, C.c_double, _D]
        L.orc_level_set_inlet.argtypes = [C.c_void_p, C.POINTER(HcCone), C.c_int]
        L.orc_level_inv_dt_at.restype = C.c_double
        L.orc_level_inv_dt_at.argtypes = [C.c_void_p, _D, C.c_double]
        L.orc_o4_level_create.restype = C.c_void_p
        L.orc_o4_level_create.argtypes = [C.c_void_p]
        L.orc_o4_level_destroy.argtypes = [C.c_void_p]
        L.orc_o4_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.orc_o4_prepare.argtypes = [C.c_void_p, _D, _D, C.c_double]
        L.orc_o4_cartesian.argtypes = [C.c_void_p, _D, _D]
        L.orc_o4_seams.argtypes = [C.c_void_p, _D]
        L.orc_o4_box_native.argtypes = [C.c_void_p, _D, _IP, _IP, C.c_int, _D, _IP, _IP, C.c_double]
        L.orc_o4_rhs.argtypes = [C.c_void_p, _D, _D, _D, C.c_double]
        L.orc_o4_reflux.argtypes = [C.c_void_p, _D, _D]
        L.orc_o4_rk4_step.argtypes = [C.c_void_p, _D, C.c_double, C.c_double]
        L.orc_o4_inv_dt.restype = C.c_double
        L.orc_o4_inv_dt.argtypes = [C.c_void_p, _D]
        _berta_signatures(L, "orc")
        L.orc_usable_primitive.argtypes = [_D]
        _orc = L
    return _orc


def _berta_signatures(L: C.CDLL, prefix: str) -> None:
    """Signatures shared by the oracle's and the reference pin's fourth-order
    pointwise exports (prefix orc_ or ref_)."""
    f = lambda name: getattr(L, f"{prefix}_{name}")  # noqa: E731
    f("berta_wenoz").argtypes = [_D, _D, _D]
    f("berta_weno3").argtypes = [_D, C.c_double, _D, _D]
    f("berta_plm").argtypes = [_D, _D, _D]
    f("berta_normalize").argtypes = [_D, C.c_int]
    f("berta_normalize").restype = C.c_double
    f("berta_jameson").argtypes = [_D, C.c_double]
    f("berta_jameson").restype = C.c_double
    f("berta_avg_to_point").argtypes = [_D, _D, C.c_double, _D]
    f("berta_flux_to_avg").argtypes = [_D, _D, C.c_double, _D]
    f("berta_select").argtypes = [_D, _D, _D, _D, C.c_double, _D, _D]
    f("berta_mapped_line").argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, C.c_int, _D]
    f("sph_to_prim_raw").argtypes = [_D, _D]
    f("prim_flux").argtypes = [_D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _D]
    f("rho_floor").restype = C.c_double
    if prefix == "orc":
        f("mapped_roe").argtypes = [_D, _D, _D, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _D]
        f("factored_roe").argtypes = [_D, _D, _D, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _D]


def ref_lib() -> C.CDLL | None:
    """The reference-header pin library, or None where it was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libhcref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_roe8.argtypes = [_D, _D, C.c_double, C.c_double, C.c_int, _D]
        L.ref_rusanov.argtypes = [_D, _D, C.c_double, _D]
        L.ref_frame.argtypes = [_D, _D, _D]
        L.ref_face_flux.argtypes = [_D, _D, _D, C.c_double, C.c_double, C.c_double, C.c_int, _D]
        L.ref_mapped_roe.argtypes = [_D, _D, _D, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _D]
        L.ref_factored_roe.argtypes = [_D, _D, _D, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _D]
        L.ref_usable_primitive.argtypes = [_D, C.c_double]
        L.ref_cone_prepare.argtypes = [_D, C.c_double, _D]
        L.ref_cone_cell.argtypes = [_D, C.c_double, C.c_double, _D, _D, C.c_double, _D]
        L.ref_cme_schedule.argtypes = [_D, _D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D]
        _berta_signatures(L, "ref")
        _ref = L
    return _ref


def make_params(**kw) -> HcParams:
    """hc_params with the configs' common settings (CGS, gamma 5/3,
    r in [21.5, 215] Rsun, radial_stretch 1.5, Powell on, entropy fix 0.3)."""
    p = HcParams()
    p.spatial_order = 2
    p.limiter = 3
    p.riemann_solver = 1
    p.divergence_cleaning = 1
    p.sun_gravity = 0
    p.init_condition_type = 1
    p.temporal_order = 4
    p.nr = 16
    p.na = 16
    p.gamma = 5.0 / 3.0
    p.entropy_fix_coeff = 0.3
    p.cfl = 0.4
    p.inner_radius = 21.5 * 6.96e10
    p.outer_radius = 215.0 * 6.96e10
    p.radial_stretch = 1.5
    p.strength = 0.0
    p.spatial_operator = 2
    p.berta_detector_type = 0
    p.berta_fallback_type = 0
    p.berta_eta_d = 0.02
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class OracleLevel:
    """A cached oracle level (one box per panel)."""

    def __init__(self, params: HcParams):
        self.params = params
        self.L = lib()
        self.h = self.L.orc_level_create(C.byref(params))
        nr, na = params.nr, params.na
        self.nv = 6 * 8 * nr * na * na
        self.ng = 6 * 8 * (nr + 4) * (na + 4) ** 2

    def __del__(self):
        try:
            self.L.orc_level_destroy(self.h)
        except Exception:
            pass

    def init(self, init: HcInit) -> np.ndarray:
        ju = np.zeros(self.nv)
        self.L.orc_level_init(self.h, C.byref(init), dptr(ju))
        return ju

    def prepare(self, ju: np.ndarray, t: float = 0.0) -> np.ndarray:
        w = np.zeros(self.ng)
        self.L.orc_level_prepare(self.h, dptr(ju), dptr(w), t)
        return w

    def inv_dt_at(self, ju: np.ndarray, t: float) -> float:
        """CFL rate with the cone density floor of the inlet active at t."""
        return self.L.orc_level_inv_dt_at(self.h, dptr(ju), t)

    def set_inlet(self, cones) -> None:
        """Cone clouds fed through the inner boundary while they cross it."""
        arr = (HcCone * max(len(cones), 1))(*cones)
        self.L.orc_level_set_inlet(self.h, arr, len(cones))

    def insert_cone(self, cone: HcCone, time: float, ju: np.ndarray) -> np.ndarray:
        """Cone volume insertion into ju (in place); returns [cells, grams]."""
        stats = np.zeros(2)
        self.L.orc_level_insert_cone(self.h, C.byref(cone), time, dptr(ju), dptr(stats))
        return stats

    def rhs(self, w: np.ndarray) -> np.ndarray:
        k = np.zeros(self.nv)
        self.L.orc_level_rhs(self.h, dptr(w), dptr(k))
        return k

    def rk4_step(self, ju: np.ndarray, dt: float, t: float = 0.0) -> None:
        self.L.orc_level_rk4_step(self.h, dptr(ju), dt, t)

    def inv_dt(self, ju: np.ndarray) -> float:
        return self.L.orc_level_inv_dt(self.h, dptr(ju))

    def valid(self, ju: np.ndarray) -> bool:
        return bool(self.L.orc_level_valid(self.h, dptr(ju)))

    def geometry(self, what: int) -> np.ndarray:
        n = self.L.orc_geometry(self.h, what, None)
        out = np.zeros(n)
        self.L.orc_geometry(self.h, what, dptr(out))
        return out

    def box_rhs(self, box: HcBox, w: np.ndarray, rhs: np.ndarray, fluxes=None, panel=None, scale=1.0):
        fl = (_D * 3)(*[dptr(f) if f is not None else None for f in fluxes]) if fluxes is not None else None
        pn = (_D * 6)(*[dptr(f) if f is not None else None for f in panel]) if panel is not None else None
        self.L.orc_box_rhs(self.h, C.byref(box), dptr(w), pn, scale, dptr(rhs), fl)

    def box_rhs_o4(self, box: HcBox, usph: np.ndarray, rhs: np.ndarray, fluxes=None, scale=1.0):
        fl = (_D * 3)(*[dptr(f) if f is not None else None for f in fluxes]) if fluxes is not None else None
        self.L.orc_box_rhs_o4(self.h, C.byref(box), dptr(usph), scale, dptr(rhs), fl)

    def box_gravity(self, box: HcBox, w: np.ndarray, rhs: np.ndarray):
        self.L.orc_box_gravity(self.h, C.byref(box), dptr(w), dptr(rhs))

    def box_gravity_o4(self, box: HcBox, usph: np.ndarray, rhs: np.ndarray):
        self.L.orc_box_gravity_o4(self.h, C.byref(box), dptr(usph), dptr(rhs))


class OracleLevelO4:
    """The fourth-order level step of the oracle: stage preparation (Cartesian
    conversion, seam ghosts, native conversion, radial ghosts), the per-panel
    operator with the seam flux register, RK4 and the CFL rate."""

    def __init__(self, params: HcParams):
        self.base = OracleLevel(params)
        self.L = self.base.L
        self.h = self.L.orc_o4_level_create(self.base.h)
        sz = (C.c_long * 5)()
        self.L.orc_o4_sizes(self.h, sz)
        self.nv, self.ng, self.nc, self.g, self.ga = (int(x) for x in sz)
        self.nr, self.na = params.nr, params.na

    def __del__(self):
        try:
            self.L.orc_o4_level_destroy(self.h)
        except Exception:
            pass

    def init(self, init: HcInit) -> np.ndarray:
        return self.base.init(init)

    def prepare(self, ju: np.ndarray, t: float = 0.0) -> np.ndarray:
        us = np.zeros(6 * 8 * self.ng)
        self.L.orc_o4_prepare(self.h, dptr(ju), dptr(us), t)
        return us

    def cartesian(self, ju: np.ndarray) -> np.ndarray:
        cart = np.zeros(6 * 8 * self.nc)
        self.L.orc_o4_cartesian(self.h, dptr(ju), dptr(cart))
        return cart

    def box_native(self, cart: np.ndarray, cart_lo, block: int, us: np.ndarray, us_lo, t: float) -> None:
        """Native averages of one box (o4BoxNative): cart [8][k][j][i] over
        cart_lo .. (its shape), us likewise over us_lo."""
        cn = (C.c_int * 3)(cart.shape[3], cart.shape[2], cart.shape[1])
        un = (C.c_int * 3)(us.shape[3], us.shape[2], us.shape[1])
        self.L.orc_o4_box_native(self.h, dptr(cart), (C.c_int * 3)(*cart_lo), cn, block, dptr(us),
                                 (C.c_int * 3)(*us_lo), un, t)

    def seams(self, cart: np.ndarray) -> None:
        self.L.orc_o4_seams(self.h, dptr(cart))

    def rhs(self, us: np.ndarray, reg: np.ndarray | None = None, weight: float = 1.0) -> np.ndarray:
        k = np.zeros(6 * 8 * self.nv)
        self.L.orc_o4_rhs(self.h, dptr(us), dptr(k), dptr(reg) if reg is not None else None, weight)
        return k

    def register(self) -> np.ndarray:
        return np.zeros(6 * 2 * 2 * 8 * self.na * self.nr)

    def reflux(self, reg: np.ndarray, ju: np.ndarray) -> None:
        self.L.orc_o4_reflux(self.h, dptr(reg), dptr(ju))

    def rk4_step(self, ju: np.ndarray, dt: float, t: float = 0.0) -> None:
        self.L.orc_o4_rk4_step(self.h, dptr(ju), dt, t)

    def inv_dt(self, ju: np.ndarray) -> float:
        return self.L.orc_o4_inv_dt(self.h, dptr(ju))


def cone_prepare(spec: HcConeSpec, inner_radius: float) -> HcCone | None:
    """The oracle's prepareConeCloud restatement (None where it fails)."""
    out = HcCone()
    return out if lib().orc_cone_prepare(C.byref(spec), inner_radius, C.byref(out)) == 0 else None


def cone_cell(cone: HcCone, time: float, pos, ambient, gamma: float):
    """(inside, delta[8]) of one cell of the oracle's cone insertion."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    amb = np.ascontiguousarray(ambient, dtype=np.float64)
    delta = np.zeros(8)
    inside = lib().orc_cone_cell(C.byref(cone), time, dptr(pos), dptr(amb), gamma, dptr(delta))
    return bool(inside), delta


def ref_cone_prepare(spec: HcConeSpec, inner_radius: float) -> np.ndarray | None:
    """The reference's prepareConeCloud (src/MHD_CME.H) compiled from source:
    [axis(3), radius, entry shift, entry time, speed, end time, insertion time]."""
    R = ref_lib()
    vec = np.array([getattr(spec, k) for k in CONE_SPEC_FIELDS])
    out = np.zeros(9)
    return out if R.ref_cone_prepare(dptr(vec), inner_radius / 6.96e10, dptr(out)) == 0 else None


def ref_cone_cell(spec: HcConeSpec, inner_radius: float, time: float, pos, ambient, gamma: float):
    """(inside, delta[8]) of the reference's sample + loadDensity + increment."""
    R = ref_lib()
    vec = np.array([getattr(spec, k) for k in CONE_SPEC_FIELDS])
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    amb = np.ascontiguousarray(ambient, dtype=np.float64)
    delta = np.zeros(8)
    rc = R.ref_cone_cell(dptr(vec), inner_radius / 6.96e10, time, dptr(pos), dptr(amb), gamma, dptr(delta))
    assert rc >= 0
    return bool(rc), delta


# ---------------------------------------------------------------------------
# AMR Runge-Kutta stage logic (numpy; every increment rounds the product,
# then the sum, as BoxData::increment does).
# advanceRungeKuttaSynchronous: src/MHD_AMRRungeKutta.H:5-41 (tableaus :9-12).
# restrictTo / Stencil::AvgDown: src/MHD_AMR.H:597-609.
# ---------------------------------------------------------------------------
RK_A = {3: ((0, 0, 0, 0), (0.5, 0, 0, 0), (-1, 2, 0, 0), (0, 0, 0, 0)),
        4: ((0, 0, 0, 0), (0.5, 0, 0, 0), (0, 0.5, 0, 0), (0, 0, 1, 0))}
RK_B = {3: (1.0 / 6, 2.0 / 3, 1.0 / 6, 0), 4: (1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6)}


def amr_rk_stage(state: np.ndarray, stage: np.ndarray, rk: list, order: int, s: int, dt: float) -> None:
    """One box: s < order writes the stage state (amrCopyValid + increments,
    :22-27); s == order updates the state in place (:37)."""
    if s < order:
        v = state.copy()
        for p in range(s):
            if RK_A[order][s][p] != 0:
                v = v + (dt * RK_A[order][s][p]) * rk[p]
        stage[...] = v
    else:
        for p in range(order):
            state[...] = state + (dt * RK_B[order][p]) * rk[p]


def amr_restrict(fine: np.ndarray, fine_lo, coarse: np.ndarray, coarse_lo, lo, hi, ratio) -> None:
    """Coarse cells lo..hi of coarse [8][n2][n1][n0] (low corner coarse_lo)
    = mean of the fine cells of fine [8][m2][m1][m0] (low corner fine_lo)
    they cover, summed radial-fastest as (1/prod ratio) * value terms."""
    w = 1.0 / float(ratio[0] * ratio[1] * ratio[2])
    I = np.arange(lo[0], hi[0] + 1)
    J = np.arange(lo[1], hi[1] + 1)
    K = np.arange(lo[2], hi[2] + 1)
    total = np.zeros((8, K.size, J.size, I.size))
    for kk in range(ratio[2]):
        for jj in range(ratio[1]):
            for ii in range(ratio[0]):
                fi = I * ratio[0] + ii - fine_lo[0]
                fj = J * ratio[1] + jj - fine_lo[1]
                fk = K * ratio[2] + kk - fine_lo[2]
                total = total + w * fine[:, fk[:, None, None], fj[None, :, None], fi[None, None, :]]
    coarse[:, K[0] - coarse_lo[2]:K[-1] - coarse_lo[2] + 1, J[0] - coarse_lo[1]:J[-1] - coarse_lo[1] + 1,
           I[0] - coarse_lo[0]:I[-1] - coarse_lo[0] + 1] = total


def amr_reflux(fine_flux, fine_lo, coarse_flux, coarse_lo, rhs, rhs_lo, lo, hi, ratio, d, fine_side, scale) -> None:
    """Reflux of coarse faces lo..hi of direction d covered by the fine level
    (src/MHD_AMR.H:651-665,916-931, the flux-register correction): for each
    face, the mean of the ratio x ratio covering fine faces (products then
    sums, the higher transverse index outer) minus the coarse face flux,
    times -scale (fine_side 1: the corrected cell is below the face) or
    +scale (fine_side 0: the cell above), added to the coarse rhs.  Arrays
    are [8][k][j][i] over boxes with the given low corners."""
    t1, t2 = [x for x in range(3) if x != d]
    w = 1.0 / float(ratio[t1] * ratio[t2])
    coef = -scale if fine_side else scale
    for K in range(lo[2], hi[2] + 1):
        for J in range(lo[1], hi[1] + 1):
            for I in range(lo[0], hi[0] + 1):
                f = [I, J, K]
                mean = np.zeros(8)
                for b2 in range(ratio[t2]):
                    for b1 in range(ratio[t1]):
                        g = [0, 0, 0]
                        g[d] = f[d] * ratio[d]
                        g[t1] = f[t1] * ratio[t1] + b1
                        g[t2] = f[t2] * ratio[t2] + b2
                        mean = mean + w * fine_flux[:, g[2] - fine_lo[2], g[1] - fine_lo[1], g[0] - fine_lo[0]]
                diff = mean - coarse_flux[:, K - coarse_lo[2], J - coarse_lo[1], I - coarse_lo[0]]
                cell = list(f)
                if fine_side:
                    cell[d] -= 1
                idx = (slice(None), cell[2] - rhs_lo[2], cell[1] - rhs_lo[1], cell[0] - rhs_lo[0])
                rhs[idx] = rhs[idx] + coef * diff


# ---------------------------------------------------------------------------
# Coarse-fine fourth-order interpolation: src/MHD_AMRInterpolation.H:39-155,
# applied to the donor data by src/MHD_AMRFourthOrder.H:27-39.
# ---------------------------------------------------------------------------
def amr_cf_inverse_moments():
    """Exact inverse (Fractions, indexed [n][i]) of the moment matrix
    A[i][n] = average of x^n over coarse cell i (centre i - 2, unit width):
    the quartic matching five cell averages has coefficients a = A^-1 u."""
    from fractions import Fraction as F
    A = []
    for i in range(5):
        c = F(i - 2)
        A.append([F(1), c, c * c + F(1, 12), c ** 3 + c / 4, c ** 4 + c * c / 2 + F(1, 80)])
    n = 5
    M = [A[r] + [F(int(r == j)) for j in range(n)] for r in range(n)]
    for col in range(n):
        piv = next(r for r in range(col, n) if M[r][col] != 0)
        M[col], M[piv] = M[piv], M[col]
        pv = M[col][col]
        M[col] = [v / pv for v in M[col]]
        for r in range(n):
            if r != col and M[r][col] != 0:
                f = M[r][col]
                M[r] = [a - f * b for a, b in zip(M[r], M[col])]
    return [[M[r][n + j] for j in range(n)] for r in range(n)]


def amr_cf_weights(ratio: int, child: int) -> np.ndarray:
    """amrFourthOrderWeights (:39-56): the child's moments in double times
    the exact inverse rounded to double, summed over the moments in order."""
    if ratio == 1:
        return np.array([0.0, 0.0, 1.0, 0.0, 0.0])
    inv = [[float(v) for v in row] for row in amr_cf_inverse_moments()]
    x = (child + 0.5) / ratio - 0.5
    h = 1.0 / ratio
    moment = [1.0, x, x * x + h * h / 12, x * x * x + x * h * h / 4,
              x * x * x * x + x * x * h * h / 2 + h * h * h * h / 80]
    w = []
    for i in range(5):
        v = 0.0
        for n in range(5):
            v += moment[n] * inv[n][i]
        w.append(v)
    return np.array(w)


def amr_cf_interpolate(coarse: np.ndarray, coarse_lo, fine: np.ndarray, fine_lo, valid_lo, valid_hi, ratio) -> None:
    """The separable passes of amrInterpolateFourthOrder (:122-155) for every
    fine storage cell outside the valid region, then the donor update of
    MHD_AMRFourthOrder.H:31-38 (finite in every component, else unchanged).
    coarse [C][k][j][i] over its box (low corner coarse_lo), fine likewise."""
    C = coarse.shape[0]
    fn = fine.shape[1:][::-1]
    cn = coarse.shape[1:][::-1]
    weights = [[amr_cf_weights(ratio[d], ch) for ch in range(ratio[d])] for d in range(3)]
    with np.errstate(all="ignore"):
        for k in range(fn[2]):
            for j in range(fn[1]):
                for i in range(fn[0]):
                    p = (fine_lo[0] + i, fine_lo[1] + j, fine_lo[2] + k)
                    if all(valid_lo[d] <= p[d] <= valid_hi[d] for d in range(3)):
                        continue
                    q = [p[d] // ratio[d] for d in range(3)]   # floor division
                    w = [weights[d][p[d] - q[d] * ratio[d]] for d in range(3)]
                    out = np.zeros(C)
                    for c in range(C):
                        value = 0.0
                        for k2 in range(-2, 3):
                            if w[2][k2 + 2] == 0:
                                continue
                            v1 = 0.0
                            for k1 in range(-2, 3):
                                if w[1][k1 + 2] == 0:
                                    continue
                                v0 = 0.0
                                for k0 in range(-2, 3):
                                    if w[0][k0 + 2] == 0:
                                        continue
                                    a = q[0] + k0 - coarse_lo[0]
                                    b = q[1] + k1 - coarse_lo[1]
                                    e = q[2] + k2 - coarse_lo[2]
                                    if not (0 <= a < cn[0] and 0 <= b < cn[1] and 0 <= e < cn[2]):
                                        v0 = float("nan")
                                        break
                                    v0 = v0 + w[0][k0 + 2] * float(coarse[c, e, b, a])
                                v1 = v1 + w[1][k1 + 2] * v0
                            value = value + w[2][k2 + 2] * v1
                        out[c] = value
                    if np.all(np.isfinite(out)):
                        fine[:, k, j, i] = out


def _at(a: np.ndarray, lo, x, c=None):
    """Value of SoA array a ([C][k][j][i] or [k][j][i]) over a box with low corner lo at point x."""
    idx = (x[2] - lo[2], x[1] - lo[1], x[0] - lo[0])
    return float(a[idx]) if c is None else float(a[(c,) + idx])


def amr_cf_mapped(jac, jac_lo, donor, donor_lo, state, state_lo, mapped, mapped_lo, valid_lo, valid_hi) -> None:
    """<JU> on valid.grow(2) (src/MHD_AMRFourthOrder.H:41-61): valid cells copy
    the state; the others J U + sum_d (J(p+e) - J(p-e)) (U(p+e) - U(p-e)) / 48."""
    mn = mapped.shape[1:][::-1]
    for k in range(mn[2]):
        for j in range(mn[1]):
            for i in range(mn[0]):
                p = (mapped_lo[0] + i, mapped_lo[1] + j, mapped_lo[2] + k)
                if all(valid_lo[d] <= p[d] <= valid_hi[d] for d in range(3)):
                    for c in range(8):
                        mapped[c, k, j, i] = _at(state, state_lo, p, c)
                    continue
                J = _at(jac, jac_lo, p)
                for c in range(8):
                    value = J * _at(donor, donor_lo, p, c)
                    for d in range(3):
                        a = list(p); b = list(p)
                        a[d] += 1; b[d] -= 1
                        dJ = _at(jac, jac_lo, a) - _at(jac, jac_lo, b)
                        value = value + dJ * (_at(donor, donor_lo, a, c) - _at(donor, donor_lo, b, c)) / 48
                    mapped[c, k, j, i] = value


def amr_cf_quotient(jac, jac_lo, mapped, mapped_lo, out, out_lo, valid_lo, valid_hi, block_lo, block_hi) -> None:
    """<U> on the valid cells (src/MHD_AMRFourthOrder.H:62-80): Q = <JU>/J,
    out = Q - (sum_d 0.5 (J(p+e) - J(p-e)) D_d Q) / (12 J), D_d the
    undivided derivative (centred; second-order one-sided on the block's
    first and last cells, the restatement of deriv3case)."""
    for k in range(valid_lo[2], valid_hi[2] + 1):
        for j in range(valid_lo[1], valid_hi[1] + 1):
            for i in range(valid_lo[0], valid_hi[0] + 1):
                p = (i, j, k)
                Jp = _at(jac, jac_lo, p)
                for c in range(8):
                    def Q(x):
                        return _at(mapped, mapped_lo, x, c) / _at(jac, jac_lo, x)
                    correction = 0.0
                    for d in range(3):
                        if p[d] == block_lo[d]:
                            base, w = p[d], (-1.5, 2.0, -0.5)
                        elif p[d] == block_hi[d]:
                            base, w = p[d] - 2, (0.5, -2.0, 1.5)
                        else:
                            base, w = p[d] - 1, (-0.5, 0.0, 0.5)
                        derivative = 0.0
                        for m in range(3):
                            x = list(p)
                            x[d] = base + m
                            derivative = derivative + w[m] * Q(x)
                        a = list(p); b = list(p)
                        a[d] += 1; b[d] -= 1
                        dj = 0.5 * (_at(jac, jac_lo, a) - _at(jac, jac_lo, b))
                        correction = correction + dj * derivative
                    out[c, k - out_lo[2], j - out_lo[1], i - out_lo[0]] = Q(p) - correction / (12.0 * Jp)


def amr_copy(src, src_lo, dst, dst_lo, lo, hi, perm, sign, shift) -> None:
    """dst(y) = src(x) over the region lo..hi, y[d] = sign[d] x[perm[d]] + shift[d]
    (the exchanges and coarse copies of src/MHD_AMRFourthOrder.H:19-24,58,83-85)."""
    for k in range(lo[2], hi[2] + 1):
        for j in range(lo[1], hi[1] + 1):
            for i in range(lo[0], hi[0] + 1):
                x = (i, j, k)
                y = [sign[d] * x[perm[d]] + shift[d] for d in range(3)]
                dst[:, y[2] - dst_lo[2], y[1] - dst_lo[1], y[0] - dst_lo[0]] = \
                    src[:, k - src_lo[2], j - src_lo[1], i - src_lo[0]]


def cme_schedule(events, time: float, feeding: float) -> tuple[float, float]:
    """(CFL fraction, Rusanov window end) of the oracle's schedule."""
    n = len(events)
    arr = (HcCmeEvent * max(n, 1))(*events)
    out = np.zeros(2)
    lib().orc_cme_schedule(arr, n, time, feeding, dptr(out))
    return float(out[0]), float(out[1])


def ref_cme_schedule(times, cloud_end, inserted: int, time: float, target: float, feeding: float):
    """The reference's CMEInsertionSchedule (finite cone sources)."""
    t = np.ascontiguousarray(times, dtype=np.float64)
    e = np.ascontiguousarray(cloud_end, dtype=np.float64)
    out = np.zeros(2)
    ref_lib().ref_cme_schedule(dptr(t), dptr(e), len(t), inserted, time, target, feeding, dptr(out))
    return float(out[0]), float(out[1])
