"""AMR Runge-Kutta stage logic on the GPU (hc_amr_plan_create,
hc_amr_rk_stage, hc_amr_restrict) against the numpy restatement in the
oracle: uneven boxes in one launch, both tableaus, every stage, and
restrictions with isotropic and radial-only ratios.  Tolerance: exact (the
device rounds every product and sum as written)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if gpu_available():
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import AmrPlan


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


SIZES = [(8, 8, 8), (12, 8, 16), (16, 16, 16), (1, 1, 1), (32, 8, 8)]


@pytest.mark.parametrize("order", [3, 4])
def test_rk_stages_match_oracle(oracle_lib, order):
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(order)
    sh = hc.Shell(hc.Params(nr=8, na=8))
    host = []
    dev = []
    for n in SIZES:
        cells = n[0] * n[1] * n[2]
        state = rng.normal(size=8 * cells) * 10.0 ** rng.integers(-20, 20, size=8 * cells)
        host.append({"state": state, "stage": np.zeros_like(state), "rk": [np.zeros_like(state) for _ in range(4)]})
        dev.append((torch.from_numpy(state.copy()).cuda(), torch.zeros(8 * cells, dtype=torch.float64, device="cuda"),
                    [torch.zeros(8 * cells, dtype=torch.float64, device="cuda") for _ in range(4)]))
    plan = AmrPlan(sh, dev)
    dt = 0.37
    for s in range(order):
        plan.rk_stage(order, s, dt)
        for h, d in zip(host, dev):
            po.amr_rk_stage(h["state"], h["stage"], h["rk"], order, s, dt)
            assert np.array_equal(d[1].cpu().numpy(), h["stage"])
            k = rng.normal(size=h["state"].size) * np.abs(h["state"]).max()
            h["rk"][s][...] = k
            d[2][s].copy_(torch.from_numpy(k))
    plan.rk_stage(order, order, dt)
    for h, d in zip(host, dev):
        po.amr_rk_stage(h["state"], h["stage"], h["rk"], order, order, dt)
        assert np.array_equal(d[0].cpu().numpy(), h["state"])
    plan.close()


def test_restrictions_match_oracle(oracle_lib):
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(9)
    sh = hc.Shell(hc.Params(nr=8, na=8))
    cases = [dict(fine_lo=(2, 4, 6), fine_n=(8, 6, 4), coarse_lo=(0, 1, 2), coarse_n=(5, 5, 5), lo=(1, 2, 3),
                  hi=(4, 4, 4), ratio=(2, 2, 2)),
             dict(fine_lo=(0, 0, 0), fine_n=(16, 4, 4), coarse_lo=(0, 0, 0), coarse_n=(8, 4, 4), lo=(0, 0, 0),
                  hi=(7, 3, 3), ratio=(2, 1, 1)),
             dict(fine_lo=(10, 0, 2), fine_n=(4, 8, 8), coarse_lo=(4, 0, 0), coarse_n=(4, 6, 6), lo=(5, 0, 1),
                  hi=(6, 3, 4), ratio=(2, 2, 2))]
    items, ref = [], []
    for c in cases:
        fine = rng.normal(size=(8, c["fine_n"][2], c["fine_n"][1], c["fine_n"][0]))
        coarse = rng.normal(size=(8, c["coarse_n"][2], c["coarse_n"][1], c["coarse_n"][0]))
        expect = coarse.copy()
        po.amr_restrict(fine, c["fine_lo"], expect, c["coarse_lo"], c["lo"], c["hi"], c["ratio"])
        d = dict(c, fine=torch.from_numpy(fine.reshape(-1).copy()).cuda(),
                 coarse=torch.from_numpy(coarse.reshape(-1).copy()).cuda())
        items.append(d)
        ref.append(expect)
    plan = AmrPlan(sh, [], items)
    plan.restrict(0, len(items))
    for d, expect in zip(items, ref):
        assert np.array_equal(d["coarse"].cpu().numpy(), expect.reshape(-1))
    plan.close()


REFLUX = [
    dict(dir=0, fine_side=1, ratio=(2, 2, 2), lo=(2, 1, 0), hi=(2, 3, 2)),
    dict(dir=1, fine_side=0, ratio=(2, 2, 2), lo=(0, 1, 1), hi=(3, 1, 2)),
    dict(dir=2, fine_side=1, ratio=(2, 1, 1), lo=(1, 0, 3), hi=(3, 2, 3)),
]


@pytest.mark.parametrize("case", REFLUX)
def test_reflux_matches_oracle(oracle_lib, case):
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(case["dir"])
    sh = hc.Shell(hc.Params(nr=8, na=8))
    d, r = case["dir"], case["ratio"]
    coarse_n = [5, 5, 5]
    coarse_n[d] += 1                      # face box
    fine_n = [10 * r[0] // 2 + 2, 10 * r[1] // 2 + 2, 10 * r[2] // 2 + 2]
    rhs_n = (5, 5, 5)
    coarse_flux = rng.normal(size=(8, coarse_n[2], coarse_n[1], coarse_n[0]))
    fine_flux = rng.normal(size=(8, fine_n[2], fine_n[1], fine_n[0]))
    rhs = rng.normal(size=(8, rhs_n[2], rhs_n[1], rhs_n[0]))
    expect = rhs.copy()
    po.amr_reflux(fine_flux, (0, 0, 0), coarse_flux, (0, 0, 0), expect, (0, 0, 0), case["lo"], case["hi"], r, d,
                  case["fine_side"], 7.5)
    t = {k: torch.from_numpy(v.reshape(-1).copy()).cuda() for k, v in
         (("fine_flux", fine_flux), ("coarse_flux", coarse_flux), ("rhs", rhs))}
    plan = AmrPlan(sh, [])
    plan.set_reflux([dict(t, fine_lo=(0, 0, 0), fine_n=fine_n, coarse_lo=(0, 0, 0), coarse_n=coarse_n,
                          rhs_lo=(0, 0, 0), rhs_n=rhs_n, lo=case["lo"], hi=case["hi"], ratio=r, dir=d,
                          fine_side=case["fine_side"], scale=7.5)])
    plan.reflux(0, 1)
    assert np.array_equal(t["rhs"].cpu().numpy(), expect.reshape(-1))
    plan.close()


def test_reflux_launch_rejects_overlapping_patches():
    _need_gpu()
    sh = hc.Shell(hc.Params(nr=8, na=8))
    flux = torch.zeros(8 * 6 * 5 * 5, dtype=torch.float64, device="cuda")
    fine = torch.zeros(8 * 12 * 12 * 12, dtype=torch.float64, device="cuda")
    rhs = torch.zeros(8 * 125, dtype=torch.float64, device="cuda")
    base = dict(fine_flux=fine, coarse_flux=flux, rhs=rhs, fine_lo=(0, 0, 0), fine_n=(12, 12, 12),
                coarse_lo=(0, 0, 0), coarse_n=(6, 5, 5), rhs_lo=(0, 0, 0), rhs_n=(5, 5, 5), ratio=(2, 2, 2),
                dir=0, fine_side=1, scale=1.0)
    plan = AmrPlan(sh, [])
    plan.set_reflux([dict(base, lo=(2, 0, 0), hi=(2, 3, 3)), dict(base, lo=(2, 2, 2), hi=(2, 4, 4))])
    with pytest.raises(hc.HcError):
        plan.reflux(0, 2)
    plan.reflux(0, 1)
    plan.reflux(1, 1)
    plan.close()


def test_cf_interpolation_matches_oracle(oracle_lib):
    """Coarse-fine fourth-order ghost interpolation (hc_amr_cf_interpolate)
    of two fine boxes in one launch, ratio 2 in every direction and 2 in the
    angular ones only, ghost cells at negative indices, a coarse box that
    does not cover every stencil and a NaN in the coarse data: bit for bit
    against the oracle, cells without data left as they were."""
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(7)
    sh = hc.Shell(hc.Params(nr=8, na=8))
    plan = AmrPlan(sh, [])
    cases = [
        # coarse_lo, coarse_n, fine_lo, fine_n, valid_lo, valid_hi, ratio
        ((-3, -3, -3), (9, 9, 8), (-3, -3, -3), (8, 8, 8), (0, 0, 0), (3, 3, 3), (2, 2, 2)),
        ((-2, -4, -4), (8, 10, 11), (-2, -5, -5), (8, 10, 10), (0, 0, 0), (3, 3, 3), (1, 2, 2)),
    ]
    host, boxes = [], []
    for b, (clo, cn, flo, fn, vlo, vhi, ratio) in enumerate(cases):
        coarse = rng.normal(size=(8, cn[2], cn[1], cn[0])) * 10.0 ** rng.integers(-3, 3, size=(8, 1, 1, 1))
        if b == 1:
            coarse[5, 4, 5, 3] = np.nan
        fine = rng.normal(size=(8, fn[2], fn[1], fn[0]))
        want = fine.copy()
        po.amr_cf_interpolate(coarse, clo, want, flo, vlo, vhi, ratio)
        dc = torch.from_numpy(coarse.copy()).cuda()
        df = torch.from_numpy(fine.copy()).cuda()
        host.append((want, fine, df))
        boxes.append({"coarse": dc, "fine": df, "coarse_lo": clo, "coarse_n": cn, "fine_lo": flo, "fine_n": fn,
                      "valid_lo": vlo, "valid_hi": vhi, "ratio": ratio, "ncomp": 8, "_keep": dc})
    plan.set_cf_interp(boxes)
    plan.cf_interpolate(0, len(boxes))
    torch.cuda.synchronize()
    for want, fine, df in host:
        got = df.cpu().numpy()
        assert np.array_equal(got, want)
        changed = np.any(got != fine, axis=0)
        assert changed.any() and not changed.all()   # some ghosts filled, valid cells and data-less ghosts kept
    plan.close()


def test_cf_interpolation_rejects_bad_boxes():
    _need_gpu()
    sh = hc.Shell(hc.Params(nr=8, na=8))
    plan = AmrPlan(sh, [])
    t = torch.zeros(8 * 64, dtype=torch.float64, device="cuda")
    good = {"coarse": t, "fine": t, "coarse_lo": (0, 0, 0), "coarse_n": (4, 4, 4), "fine_lo": (0, 0, 0),
            "fine_n": (4, 4, 4), "valid_lo": (1, 1, 1), "valid_hi": (2, 2, 2), "ratio": (2, 2, 2), "ncomp": 8}
    for key, value in (("ratio", (9, 2, 2)), ("ncomp", 17), ("fine_n", (0, 4, 4))):
        with pytest.raises(hc.HcError):
            plan.set_cf_interp([dict(good, **{key: value})])
    plan.set_cf_interp([good, dict(good, fine=torch.zeros(8 * 64, dtype=torch.float64, device="cuda"))])
    with pytest.raises(hc.HcError):
        plan.set_cf_interp([good, good])
        plan.cf_interpolate(0, 2)                     # both write the same fine region
    plan.close()


def test_cf_fine_recovery_matches_oracle(oracle_lib):
    """<JU> of the ghost cells (hc_amr_cf_mapped) and <U> of the valid cells
    (hc_amr_cf_quotient) of two fine boxes in one launch each, one touching
    its block's low radial end and one its high angular end: bit for bit
    against the oracle."""
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(11)
    sh = hc.Shell(hc.Params(nr=8, na=8))
    plan = AmrPlan(sh, [])
    cases = [((0, 2, 3), (5, 6, 6), (0, -20, -20), (40, 40, 40)),
             ((4, -3, 1), (9, 2, 4), (-20, -20, -20), (40, 2, 40))]
    host, boxes = [], []
    for vlo, vhi, blo, bhi in cases:
        vn = [vhi[d] - vlo[d] + 1 for d in range(3)]
        g3lo = [v - 3 for v in vlo]
        g3n = [n + 6 for n in vn]
        g2lo = [v - 2 for v in vlo]
        g2n = [n + 4 for n in vn]
        jac = 1.0 + rng.random(g3n[::-1])
        donor = rng.normal(size=[8] + g3n[::-1])
        state = rng.normal(size=[8] + vn[::-1])
        want_m = np.zeros([8] + g2n[::-1])
        want_o = np.zeros([8] + vn[::-1])
        po.amr_cf_mapped(jac, g3lo, donor, g3lo, state, vlo, want_m, g2lo, vlo, vhi)
        po.amr_cf_quotient(jac, g3lo, want_m, g2lo, want_o, vlo, vlo, vhi, blo, bhi)
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
             (("jac", jac), ("donor", donor), ("state", state))}
        t["mapped"] = torch.zeros(want_m.size, dtype=torch.float64, device="cuda")
        t["out"] = torch.zeros(want_o.size, dtype=torch.float64, device="cuda")
        host.append((want_m, want_o, t))
        boxes.append(dict(t, jac_lo=g3lo, jac_n=g3n, donor_lo=g3lo, donor_n=g3n, state_lo=vlo, state_n=vn,
                          mapped_lo=g2lo, mapped_n=g2n, out_lo=vlo, out_n=vn, valid_lo=vlo, valid_hi=vhi,
                          block_lo=blo, block_hi=bhi))
    plan.set_cf_fine(boxes)
    plan.cf_mapped(0, 2)
    plan.cf_quotient(0, 2)
    torch.cuda.synchronize()
    for want_m, want_o, t in host:
        assert np.array_equal(t["mapped"].cpu().numpy().reshape(want_m.shape), want_m)
        assert np.array_equal(t["out"].cpu().numpy().reshape(want_o.shape), want_o)
    bad = dict(boxes[0], mapped_n=[n + 1 for n in boxes[0]["mapped_n"]])
    with pytest.raises(hc.HcError):
        plan.set_cf_fine([bad])
    plan.close()


def test_region_copies_match_oracle(oracle_lib):
    """hc_amr_copy: an in-panel ghost exchange between two boxes and a
    cross-panel copy with a signed axis permutation, one launch; a launch
    whose write overlaps another copy's read, or that writes memory another
    base pointer of the launch reaches, is refused."""
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(5)
    sh = hc.Shell(hc.Params(nr=8, na=8))
    plan = AmrPlan(sh, [])
    a = rng.normal(size=(8, 10, 10, 10))      # box A over -1 .. 8 (1 ghost around 0 .. 7)
    b = rng.normal(size=(8, 10, 10, 10))      # box B over 7 .. 16 along i, -1 .. 8 otherwise
    c = rng.normal(size=(8, 6, 8, 4))         # another panel's array over (0..3, 0..7, 0..5)
    ta, tb, tc = (torch.from_numpy(x.copy()).cuda() for x in (a, b, c))
    copies = [
        # B's low ghost layer (i = 7) from A's valid i = 7
        dict(src=ta, dst=tb, src_lo=(-1, -1, -1), src_n=(10, 10, 10), dst_lo=(7, -1, -1), dst_n=(10, 10, 10),
             lo=(7, 0, 0), hi=(7, 7, 7), perm=(0, 1, 2), sign=(1, 1, 1), shift=(0, 0, 0), ncomp=8),
        # A's high ghost layer (i = 8) from B's valid i = 8
        dict(src=tb, dst=ta, src_lo=(7, -1, -1), src_n=(10, 10, 10), dst_lo=(-1, -1, -1), dst_n=(10, 10, 10),
             lo=(8, 0, 0), hi=(8, 7, 7), perm=(0, 1, 2), sign=(1, 1, 1), shift=(0, 0, 0), ncomp=8),
        # C's layer k = 0 into A's low k ghost layer with a signed permutation:
        # y = (j, 3 - i, k - 1), i.e. A cells (0..7, 0..3, -1)
        dict(src=tc, dst=ta, src_lo=(0, 0, 0), src_n=(4, 8, 6), dst_lo=(-1, -1, -1), dst_n=(10, 10, 10),
             lo=(0, 0, 0), hi=(3, 7, 0), perm=(1, 0, 2), sign=(1, -1, 1), shift=(0, 3, -1), ncomp=8),
    ]
    plan.set_copies(copies)
    plan.copy(0, 3)
    torch.cuda.synchronize()
    wa, wb = a.copy(), b.copy()
    po.amr_copy(a, (-1, -1, -1), wb, (7, -1, -1), (7, 0, 0), (7, 7, 7), (0, 1, 2), (1, 1, 1), (0, 0, 0))
    po.amr_copy(b, (7, -1, -1), wa, (-1, -1, -1), (8, 0, 0), (8, 7, 7), (0, 1, 2), (1, 1, 1), (0, 0, 0))
    po.amr_copy(c, (0, 0, 0), wa, (-1, -1, -1), (0, 0, 0), (3, 7, 0), (1, 0, 2), (1, -1, 1), (0, 3, -1))
    assert np.array_equal(ta.cpu().numpy(), wa)
    assert np.array_equal(tb.cpu().numpy(), wb)
    # a copy writing A's valid cells while another reads them: refused
    racy = dict(copies[0], src=tb, dst=ta, src_lo=(7, -1, -1), dst_lo=(-1, -1, -1), lo=(8, 0, 0), hi=(8, 7, 7),
                shift=(-1, 0, 0))
    plan.set_copies([copies[0], racy])
    with pytest.raises(hc.HcError):
        plan.copy(0, 2)
    # a destination that is a sub-view of A (another base pointer into the
    # same memory) written in the same launch as A: refused
    alias = dict(copies[2], dst=ta.view(-1)[4000:], ncomp=4)
    plan.set_copies([copies[1], alias])
    with pytest.raises(hc.HcError):
        plan.copy(0, 2)
    plan.close()


def test_native_conversion_of_boxes_matches_oracle(oracle_lib):
    """hc_amr_native: native averages and radial ghosts of three fine boxes
    in one launch (one reaching into the inner radial ghosts, one into the
    outer, one inside), from random Cartesian averages, against the
    oracle's o4BoxNative.  Tolerance 1e-13 of each component's largest
    magnitude: the device contracts a*b+c into FMA where the oracle does
    not."""
    _need_gpu()
    po = oracle_lib
    rng = np.random.default_rng(23)
    params = hc.Params(nr=12, na=16, spatial_order=4, riemann_solver=2, berta_fallback_type=0)
    sh = hc.Shell(params)
    orc = po.OracleLevelO4(po.make_params(nr=12, na=16, spatial_order=4, riemann_solver=2, berta_fallback_type=0))
    plan = AmrPlan(sh, [])
    # (block, usph_lo, usph_hi): the operator's input boxes valid.grow(5)
    cases = [(0, (-5, 1, 2), (6, 12, 9)), (3, (5, 3, 4), (16, 10, 11)), (5, (2, 5, 6), (9, 10, 13))]
    host, boxes = [], []
    for b, ulo, uhi in cases:
        un = [uhi[d] - ulo[d] + 1 for d in range(3)]
        clo = [max(ulo[0], 0), ulo[1] - 1, ulo[2] - 1]
        chi = [min(uhi[0], 11), uhi[1] + 1, uhi[2] + 1]
        cn = [chi[d] - clo[d] + 1 for d in range(3)]
        cart = rng.normal(size=[8] + cn[::-1])
        cart[0] = 1.0 + rng.random(cn[::-1])
        want = np.zeros([8] + un[::-1])
        orc.box_native(cart, clo, b, want, ulo, 0.0)
        dc = torch.from_numpy(cart).cuda()
        du = torch.zeros(want.size, dtype=torch.float64, device="cuda")
        host.append((want, du))
        boxes.append({"cart": dc, "usph": du, "cart_lo": clo, "cart_n": cn, "usph_lo": ulo, "usph_n": un,
                      "block": b, "_keep": dc})
    plan.set_native(boxes)
    plan.native(0, len(boxes), 0.0)
    torch.cuda.synchronize()
    for want, du in host:
        got = du.cpu().numpy().reshape(want.shape)
        scale = np.abs(want).reshape(8, -1).max(axis=1)
        err = np.abs(got - want).reshape(8, -1).max(axis=1) / np.maximum(scale, 1e-300)
        assert np.isfinite(got).all() and (err <= 1e-13).all(), err
    # a cart box that misses a neighbour the conversion reads is refused
    bad = dict(boxes[2], cart_lo=[boxes[2]["cart_lo"][0], boxes[2]["cart_lo"][1] + 1, boxes[2]["cart_lo"][2]])
    plan.set_native([bad])
    with pytest.raises(hc.HcError):
        plan.native(0, 1, 0.0)
    plan.close()
