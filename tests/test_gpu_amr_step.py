"""A whole two-level AMR RK4 step of the fourth-order scheme on the device
(heliocubed_b200.amr.AmrStep: advanceRungeKuttaSynchronous with
prepareFourthOrder and evaluate, src/MHD_AMRRungeKutta.H:5-41,
src/MHD_AMRFourthOrder.H:5-100, src/MHD_AMR.H:1417-1499) against the same
step composed from the oracle: its level preparation and operator with the
per-evaluation panel-seam reconciliation, its box operator, native
conversion, coarse-fine interpolation, fine-box recovery, region copies,
reflux, restriction and RK tableau.

Levels: a 24 x 16^2 x 6 coarse shell and three 8^3 fine boxes of the
48 x 32^2 x 6 level (two abutting boxes on one panel, one on another) on
the perturbed wind.  Tolerance: 1e-10 per component, normwise
(max |gpu - oracle| / max |oracle|), since the device contracts a*b+c into
FMA where the oracle does not."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200 import amr
    from heliocubed_b200 import level as hl

KW = dict(spatial_order=4, riemann_solver=2, divergence_cleaning=1, sun_gravity=0, berta_fallback_type=0, cfl=0.4)
BOXES = [(0, (12, 8, 8), (19, 15, 15)), (0, (20, 8, 8), (27, 15, 15)), (3, (14, 10, 12), (21, 17, 19))]
SEED = 20261204


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _wind(orc, nr, na):
    det = orc.base.geometry(4).reshape(6, na, na)
    vol = orc.base.geometry(0).reshape(nr + 1, 4)[:nr, 3]
    return np.ascontiguousarray(hl.perturbed_wind_state(hl.Params(nr=nr, na=na, **KW), det, vol, seed=SEED)
                                .reshape(-1))


def _grow(lo, hi, w):
    return [x - w for x in lo], [hi[d] - lo[d] + 1 + 2 * w for d in range(3)]


def _zeros(n):
    return np.zeros([8] + list(n)[::-1])


def _oracle_step(po, oc, of, step, ju_c, states_f, dt, t):
    """The device step's sequence with the oracle's pieces (numpy arrays
    [8][k][j][i] over each box; the coarse level in level layout)."""
    nr, na = oc.nr, oc.na
    nA, nG = na + 12, na + 10
    pan = lambda a: a.reshape(6, 8, na, na, nr)  # noqa: E731
    nf = len(BOXES)
    state_c, stage_c = ju_c.copy(), np.zeros_like(ju_c)
    rk_c = [np.zeros_like(ju_c) for _ in range(4)]
    vn = [[hi[d] - lo[d] + 1 for d in range(3)] for _, lo, hi in BOXES]
    state_f = [s.copy() for s in states_f]
    stage_f = [np.zeros_like(s) for s in state_f]
    rk_f = [[np.zeros_like(s) for _ in range(4)] for s in state_f]
    jac = [step.f["jac"][1][q].cpu().numpy().reshape(list(_grow(lo, hi, 3)[1])[::-1])
           for q, (b, lo, hi) in enumerate(BOXES)]
    triples = [(b, lo, hi) for b, lo, hi in BOXES]
    block_hi = (2 * nr - 1, 2 * na - 1, 2 * na - 1)

    def restrict(fine, coarse):
        for q, (b, lo, hi) in enumerate(BOXES):
            po.amr_restrict(fine[q], lo, pan(coarse)[b], (0, 0, 0), [x // 2 for x in lo], [x // 2 for x in hi],
                            (2, 2, 2))

    def exchange(arrs, w):
        for cp in hl.amr_exchange_copies(triples, w):
            s, d = cp["src_box"], cp["dst_box"]
            po.amr_copy(arrs[s], _grow(BOXES[s][1], BOXES[s][2], w)[0], arrs[d],
                        _grow(BOXES[d][1], BOXES[d][2], w)[0], cp["lo"], cp["hi"], cp["perm"], cp["sign"],
                        cp["shift"])

    for s in range(4):
        po.amr_rk_stage(state_c, stage_c, rk_c, 4, s, dt)
        for q in range(nf):
            po.amr_rk_stage(state_f[q], stage_f[q], rk_f[q], 4, s, dt)
        restrict(stage_f, stage_c)
        ts = t + amr.C4[s] * dt
        us_c = oc.prepare(stage_c, ts)
        cart = oc.cartesian(stage_c).reshape(6, 8, nA, nA, nr)
        donor, mapped, out, usph = [], [], [], []
        for q, (b, lo, hi) in enumerate(BOXES):
            dl, dn = _grow(lo, hi, 6)
            ml, mn = _grow(lo, hi, 2)
            donor.append(_zeros(dn))
            po.amr_cf_interpolate(cart[b], (0, -6, -6), donor[q], dl, lo, hi, (2, 2, 2))
            mapped.append(_zeros(mn))
            po.amr_cf_mapped(jac[q], _grow(lo, hi, 3)[0], donor[q], dl, stage_f[q], lo, mapped[q], ml, lo, hi)
        exchange(mapped, 2)
        for q, (b, lo, hi) in enumerate(BOXES):
            out.append(_zeros(vn[q]))
            po.amr_cf_quotient(jac[q], _grow(lo, hi, 3)[0], mapped[q], _grow(lo, hi, 2)[0], out[q], lo, lo, hi,
                               (0, 0, 0), block_hi)
            po.amr_copy(out[q], lo, donor[q], _grow(lo, hi, 6)[0], lo, hi, (0, 1, 2), (1, 1, 1), (0, 0, 0))
        exchange(donor, 6)
        for q, (b, lo, hi) in enumerate(BOXES):
            ul, un = _grow(lo, hi, 5)
            usph.append(_zeros(un))
            of.box_native(donor[q], _grow(lo, hi, 6)[0], b, usph[q], ul, ts)
        # coarse evaluation: seams reconciled in k; each panel's own fluxes
        reg = oc.register()
        k_c = oc.rhs(us_c, reg, 1.0)
        oc.reflux(reg, k_c)
        flux_c = [np.zeros((6, 8, na + (d == 2), na + (d == 1), nr + (d == 0))) for d in range(3)]
        for b in range(6):
            box = po.HcBox()
            for d in range(3):
                box.lo[d], box.hi[d] = 0, (nr if d == 0 else na) - 1
            box.ghost, box.block = 5, b
            scratch = np.zeros(8 * nr * na * na)
            fl = [np.zeros(8 * (nr + (d == 0)) * (na + (d == 1)) * (na + (d == 2))) for d in range(3)]
            oc.base.box_rhs_o4(box, np.ascontiguousarray(us_c.reshape(6, -1)[b]), scratch, fl)
            for d in range(3):
                flux_c[d][b] = fl[d].reshape(flux_c[d][b].shape)
        k_f, flux_f = [], []
        for q, (b, lo, hi) in enumerate(BOXES):
            box = po.HcBox()
            for d in range(3):
                box.lo[d], box.hi[d] = lo[d], hi[d]
            box.ghost, box.block = 5, b
            k = np.zeros(8 * int(np.prod(vn[q])))
            fl = [np.zeros(8 * (vn[q][0] + (d == 0)) * (vn[q][1] + (d == 1)) * (vn[q][2] + (d == 2)))
                  for d in range(3)]
            of.base.box_rhs_o4(box, np.ascontiguousarray(usph[q].reshape(-1)), k, fl)
            k_f.append(k.reshape(_zeros(vn[q]).shape))
            flux_f.append([fl[d].reshape([8] + [vn[q][e] + (e == d) for e in range(3)][::-1]) for d in range(3)])
        kc = pan(k_c)
        for p in step.patches:
            q, b, d = p["box"], p["panel"], p["dir"]
            po.amr_reflux(flux_f[q][d], BOXES[q][1], flux_c[d][b], (0, 0, 0), kc[b], (0, 0, 0), p["lo"], p["hi"],
                          (2, 2, 2), d, p["fine_side"], p["scale"])
        restrict(k_f, k_c)
        rk_c[s] = k_c.copy()
        for q in range(nf):
            rk_f[q][s] = k_f[q].copy()
    po.amr_rk_stage(state_c, stage_c, rk_c, 4, 4, dt)
    for q in range(nf):
        po.amr_rk_stage(state_f[q], stage_f[q], rk_f[q], 4, 4, dt)
    restrict(state_f, state_c)
    return state_c, state_f


def test_two_level_amr_step_matches_oracle(oracle_lib):
    _need_gpu()
    po = oracle_lib
    nrc, nac = 24, 16
    coarse = hc.Shell(hc.Params(nr=nrc, na=nac, **KW))
    fine = hc.Shell(hc.Params(nr=2 * nrc, na=2 * nac, **KW))
    oc = po.OracleLevelO4(po.make_params(nr=nrc, na=nac, **KW))
    of = po.OracleLevelO4(po.make_params(nr=2 * nrc, na=2 * nac, **KW))
    ju_c = _wind(oc, nrc, nac)
    ju_f = _wind(of, 2 * nrc, 2 * nac).reshape(6, 8, 2 * nac, 2 * nac, 2 * nrc)
    states_f = [np.ascontiguousarray(ju_f[b][:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1])
                for b, lo, hi in BOXES]
    dt = 0.4 / max(oc.inv_dt(ju_c), of.inv_dt(np.ascontiguousarray(ju_f.reshape(-1))))
    step = amr.AmrStep(coarse, fine, BOXES)
    step.load(torch.from_numpy(ju_c).cuda(), [torch.from_numpy(s).cuda() for s in states_f])
    step.step(dt, 0.0)
    torch.cuda.synchronize()
    want_c, want_f = _oracle_step(po, oc, of, step, ju_c, states_f, dt, 0.0)
    got_c = step.state_c.cpu().numpy()
    assert np.isfinite(got_c).all()
    err = rel_err_components(got_c.reshape(6, 8, -1), want_c.reshape(6, 8, -1))
    assert err.max() <= 1e-10, err
    for q in range(len(BOXES)):
        got = step.fine_state(q).cpu().numpy().reshape(8, -1)
        err = rel_err_components(got, want_f[q].reshape(8, -1), 0)
        assert np.isfinite(got).all() and err.max() <= 1e-10, (q, err)
    # the step moved both levels, and the covered coarse cells hold the
    # restriction of the fine boxes
    assert not np.array_equal(got_c, ju_c)
    step.close()


def test_amr_step_refuses_boxes_out_of_scope():
    _need_gpu()
    coarse = hc.Shell(hc.Params(nr=24, na=16, **KW))
    fine = hc.Shell(hc.Params(nr=48, na=32, **KW))
    for bad in ([(0, (13, 8, 8), (20, 15, 15))],            # not aligned to the refinement
                [(0, (2, 8, 8), (9, 15, 15))],              # next to the inner boundary
                [(0, (12, 0, 8), (19, 7, 15))],             # donor ghosts across a panel edge
                [(0, (12, 8, 8), (19, 15, 15)), (0, (18, 8, 8), (25, 15, 15))]):   # overlapping
        with pytest.raises(ValueError):
            amr.AmrStep(coarse, fine, bad)
