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
