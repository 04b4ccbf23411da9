"""Coarse-fine fourth-order interpolation (src/MHD_AMRInterpolation.H:39-155,
src/MHD_AMRFourthOrder.H:27-39) on the CPU: the weights the library
computes on the host (hc_amr_cf_weights) against the oracle's, bit for bit;
the exact properties of the oracle's weights; and the oracle's
interpolation on data it must reproduce."""
import sys
from fractions import Fraction as F
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from oracle import pyoracle as po  # noqa: E402


def _exact_weights(ratio, child):
    """Exact rational weights: child moments (exact) times the exact inverse."""
    inv = po.amr_cf_inverse_moments()
    h = F(1, ratio)
    x = F(2 * child + 1, 2 * ratio) - F(1, 2)
    moment = [F(1), x, x * x + h * h / 12, x ** 3 + x * h * h / 4, x ** 4 + x * x * h * h / 2 + h ** 4 / 80]
    return [sum(moment[n] * inv[n][i] for n in range(5)) for i in range(5)]


def test_library_weights_match_oracle(product_lib_path):
    from heliocubed_b200.level import amr_cf_weights
    for ratio in range(1, 9):
        for child in range(ratio):
            assert np.array_equal(amr_cf_weights(ratio, child), po.amr_cf_weights(ratio, child)), (ratio, child)


def test_bad_weight_arguments_rejected(product_lib_path):
    from heliocubed_b200 import HcError
    from heliocubed_b200.level import amr_cf_weights
    for ratio, child in ((0, 0), (9, 0), (2, 2), (2, -1)):
        with pytest.raises(HcError):
            amr_cf_weights(ratio, child)


@pytest.mark.parametrize("ratio", [2, 3, 4])
def test_exact_weight_properties(ratio):
    ws = [_exact_weights(ratio, c) for c in range(ratio)]
    # each child's weights sum to one; the children average to the parent
    for w in ws:
        assert sum(w) == 1
    for i in range(5):
        assert sum(w[i] for w in ws) / ratio == (1 if i == 2 else 0)
    # quartics are reproduced exactly: child average of x^n from the five
    # coarse averages of x^n
    inv_cells = [(F(i - 2) - F(1, 2), F(i - 2) + F(1, 2)) for i in range(5)]
    for n in range(5):
        coarse = [(b ** (n + 1) - a ** (n + 1)) / (n + 1) / (b - a) for a, b in inv_cells]
        for c, w in enumerate(ws):
            a = F(c, ratio) - F(1, 2)
            b = a + F(1, ratio)
            assert sum(wi * ui for wi, ui in zip(w, coarse)) == (b ** (n + 1) - a ** (n + 1)) / (n + 1) / (b - a)
    # the double weights are the exact ones rounded
    for c in range(ratio):
        assert np.max(np.abs(po.amr_cf_weights(ratio, c) - np.array([float(v) for v in ws[c]]))) < 1e-15


def _cell_avg_cubic(lo, hi, coef):
    """Average over [lo, hi] of the product polynomial sum_n coef[d][n] x^n per direction."""
    out = 1.0
    for d in range(3):
        a, b = lo[d], hi[d]
        out *= sum(c * (b ** (n + 1) - a ** (n + 1)) / (n + 1) for n, c in enumerate(coef[d])) / (b - a)
    return out


def test_oracle_interpolation_reproduces_quartics():
    # coarse averages of a product of quartics; the fine ghost cells must
    # get the fine averages (ratio 2, negative fine indices included)
    coef = [[0.3, -0.2, 0.1, 0.05, -0.01], [1.0, 0.1, -0.05, 0.02, 0.003], [0.5, 0.0, 0.02, -0.01, 0.002]]
    clo, cn = (-4, -4, -4), (12, 12, 12)
    coarse = np.zeros((1, cn[2], cn[1], cn[0]))
    for k in range(cn[2]):
        for j in range(cn[1]):
            for i in range(cn[0]):
                c = (clo[0] + i, clo[1] + j, clo[2] + k)
                coarse[0, k, j, i] = _cell_avg_cubic([x * 1.0 for x in c], [x + 1.0 for x in c], coef)
    flo, fn = (-2, -2, -2), (8, 8, 8)
    fine = np.full((1, fn[2], fn[1], fn[0]), -7.0)
    po.amr_cf_interpolate(coarse, clo, fine, flo, (0, 0, 0), (3, 3, 3), (2, 2, 2))
    for k in range(fn[2]):
        for j in range(fn[1]):
            for i in range(fn[0]):
                p = (flo[0] + i, flo[1] + j, flo[2] + k)
                if all(0 <= p[d] <= 3 for d in range(3)):
                    assert fine[0, k, j, i] == -7.0      # valid cells untouched
                    continue
                want = _cell_avg_cubic([x / 2 for x in p], [(x + 1) / 2 for x in p], coef)
                assert abs(fine[0, k, j, i] - want) < 1e-12 * (1 + abs(want))


def test_oracle_leaves_cells_without_coarse_data():
    coarse = np.ones((2, 5, 5, 5))
    coarse[1, 2, 2, 2] = np.nan
    fine = np.full((2, 4, 4, 4), 3.0)
    # coarse box 0..4 in each direction; fine cells 0..3 (parents 0, 1) need
    # coarse -2 .. 3: outside on the low side, so nothing is written
    po.amr_cf_interpolate(coarse, (0, 0, 0), fine, (0, 0, 0), (1, 1, 1), (0, 0, 0), (2, 2, 2))
    assert np.all(fine == 3.0)
    # shifted so every stencil is inside, the NaN poisons only the cells
    # whose stencils reach it with nonzero weight
    fine2 = np.full((2, 2, 2, 2), 3.0)
    po.amr_cf_interpolate(coarse, (-2, -2, -2), fine2, (0, 0, 0), (1, 1, 1), (0, 0, 0), (2, 2, 2))
    assert np.all(fine2 == 3.0)    # every fine cell here reads coarse (0, 0, 0) = the NaN
    coarse[1, 2, 2, 2] = 1.0
    po.amr_cf_interpolate(coarse, (-2, -2, -2), fine2, (0, 0, 0), (1, 1, 1), (0, 0, 0), (2, 2, 2))
    assert np.allclose(fine2, 1.0, rtol=0, atol=1e-14)


def _fine_case(rng, valid_lo, valid_hi, jac_fn, u_fn):
    """Arrays of one fine box: J and the donor on valid.grow(3), the state
    <JU> on valid, the mapped box valid.grow(2)."""
    g3lo = [v - 3 for v in valid_lo]
    g3n = [valid_hi[d] - valid_lo[d] + 7 for d in range(3)]
    jac = np.zeros(g3n[::-1])
    donor = np.zeros([8] + g3n[::-1])
    for k in range(g3n[2]):
        for j in range(g3n[1]):
            for i in range(g3n[0]):
                x = (g3lo[0] + i, g3lo[1] + j, g3lo[2] + k)
                jac[k, j, i] = jac_fn(x)
                donor[:, k, j, i] = u_fn(x)
    vn = [valid_hi[d] - valid_lo[d] + 1 for d in range(3)]
    state = rng.normal(size=[8] + vn[::-1])
    g2lo = [v - 2 for v in valid_lo]
    mapped = np.zeros([8] + [n + 4 for n in vn][::-1])
    return g3lo, jac, donor, state, g2lo, mapped


def test_oracle_fine_recovery_is_exact_for_constant_and_linear_data():
    rng = np.random.default_rng(3)
    vlo, vhi = (0, 0, 0), (3, 3, 3)
    block_lo, block_hi = (0, -10, -10), (20, 20, 20)     # the radial block starts at the valid box
    # constant J: the product and quotient corrections vanish
    g3lo, jac, donor, state, g2lo, mapped = _fine_case(rng, vlo, vhi, lambda x: 2.0, lambda x: np.arange(8) + 1.0)
    po.amr_cf_mapped(jac, g3lo, donor, g3lo, state, vlo, mapped, g2lo, vlo, vhi)
    assert np.array_equal(mapped[:, 2:6, 2:6, 2:6], state)            # valid cells copy the state
    ghost = np.ones(mapped.shape[1:], bool)
    ghost[2:6, 2:6, 2:6] = False
    assert np.all(mapped[:, ghost] == 2.0 * (np.arange(8) + 1.0)[:, None])
    out = np.zeros((8, 4, 4, 4))
    po.amr_cf_quotient(jac, g3lo, mapped, g2lo, out, vlo, vlo, vhi, block_lo, block_hi)
    assert np.array_equal(out, state / 2.0)
    # linear J, constant U: <JU> = J U exactly, and the quotient returns U
    g3lo, jac, donor, state, g2lo, mapped = _fine_case(rng, vlo, vhi, lambda x: 1.0 + 0.25 * x[0] + 0.125 * x[1],
                                                       lambda x: np.full(8, 3.0))
    state[...] = 0.0
    for k in range(4):
        for j in range(4):
            for i in range(4):
                state[:, k, j, i] = 3.0 * (1.0 + 0.25 * i + 0.125 * j)
    po.amr_cf_mapped(jac, g3lo, donor, g3lo, state, vlo, mapped, g2lo, vlo, vhi)
    po.amr_cf_quotient(jac, g3lo, mapped, g2lo, out, vlo, vlo, vhi, block_lo, block_hi)
    assert np.max(np.abs(out - 3.0)) < 1e-14


def test_oracle_fine_quotient_is_fourth_order():
    # smooth J and U: the quotient of the exact product averages recovers
    # the exact U averages to O(h^4) (h the cell width in units of the data)
    def case(h):
        def avg(f, x):
            # Gauss-Legendre 3 points per direction over the cell [x, x + 1] * h
            g = (0.5 - np.sqrt(15) / 10, 0.5, 0.5 + np.sqrt(15) / 10)
            wts = (5 / 18, 8 / 18, 5 / 18)
            tot = 0.0
            for a, wa in zip(g, wts):
                for b, wb in zip(g, wts):
                    for c, wc in zip(g, wts):
                        tot = tot + wa * wb * wc * f(((x[0] + a) * h, (x[1] + b) * h, (x[2] + c) * h))
            return tot
        Jf = lambda y: 1.0 + 0.3 * np.sin(y[0] + 0.5 * y[1]) + 0.2 * y[2] * y[2]
        Uf = lambda y: np.cos(y[0] - y[2]) + 0.5 * y[1]
        vlo, vhi = (0, 0, 0), (1, 1, 1)
        g3lo, jac, donor, state, g2lo, mapped = _fine_case(np.random.default_rng(0), vlo, vhi,
                                                           lambda x: avg(Jf, x), lambda x: np.full(8, avg(Uf, x)))
        for k in range(2):
            for j in range(2):
                for i in range(2):
                    state[:, k, j, i] = avg(lambda y: Jf(y) * Uf(y), (i, j, k))
        # ghosts from the donor's U averages, valid from the exact <JU>
        po.amr_cf_mapped(jac, g3lo, donor, g3lo, state, vlo, mapped, g2lo, vlo, vhi)
        out = np.zeros((8, 2, 2, 2))
        po.amr_cf_quotient(jac, g3lo, mapped, g2lo, out, vlo, vlo, vhi, (-50, -50, -50), (50, 50, 50))
        exact = np.array([[[avg(Uf, (i, j, k)) for i in range(2)] for j in range(2)] for k in range(2)])
        return np.max(np.abs(out[0] - exact))
    e1, e2 = case(0.2), case(0.1)
    assert e1 / e2 > 12.0, (e1, e2)


def test_exchange_copies_fill_ghosts_from_neighbours():
    """amr_exchange_copies on three boxes of one panel (and one on another
    panel): applied with the oracle's region copy, every ghost cell covered
    by a neighbour's valid cells gets the neighbour's value of a global
    field; ghosts outside every neighbour keep their fill; no valid cell is
    written."""
    from heliocubed_b200.level import amr_exchange_copies
    g = 2
    boxes = [(0, (0, 0, 0), (3, 3, 3)), (0, (4, 0, 0), (7, 3, 3)), (0, (0, 4, 0), (3, 7, 3)), (1, (4, 0, 0), (7, 3, 3))]
    field = lambda x: 1000.0 * x[0] + 100.0 * x[1] + 10.0 * x[2]
    arrays = []
    for panel, lo, hi in boxes:
        n = [hi[d] - lo[d] + 1 + 2 * g for d in range(3)]
        a = np.full((1, n[2], n[1], n[0]), -1.0)
        for k in range(lo[2], hi[2] + 1):
            for j in range(lo[1], hi[1] + 1):
                for i in range(lo[0], hi[0] + 1):
                    a[0, k - lo[2] + g, j - lo[1] + g, i - lo[0] + g] = field((i, j, k)) + 1e6 * panel
        arrays.append(a)
    before = [a.copy() for a in arrays]
    copies = amr_exchange_copies(boxes, g)
    assert all(boxes[c["src_box"]][0] == boxes[c["dst_box"]][0] for c in copies)
    for c in copies:
        sb, db = boxes[c["src_box"]], boxes[c["dst_box"]]
        po.amr_copy(before[c["src_box"]], [v - g for v in sb[1]], arrays[c["dst_box"]], [v - g for v in db[1]],
                    c["lo"], c["hi"], c["perm"], c["sign"], c["shift"])
    for b, (panel, lo, hi) in enumerate(boxes):
        a = arrays[b]
        n = a.shape[1:][::-1]
        for k in range(n[2]):
            for j in range(n[1]):
                for i in range(n[0]):
                    x = (lo[0] - g + i, lo[1] - g + j, lo[2] - g + k)
                    valid = all(lo[d] <= x[d] <= hi[d] for d in range(3))
                    owner = [q for q, (pq, ql, qh) in enumerate(boxes)
                             if pq == panel and all(ql[d] <= x[d] <= qh[d] for d in range(3))]
                    if valid:
                        assert a[0, k, j, i] == before[b][0, k, j, i]
                    elif owner:
                        assert a[0, k, j, i] == field(x) + 1e6 * panel
                    else:
                        assert a[0, k, j, i] == -1.0
