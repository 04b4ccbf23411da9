"""Batched fourth-order operator (hc_o4_batch_*): boxes of different sizes,
panels and positions evaluated with one launch per operator kernel give the
same rhs and fluxes as one hc_box_rhs_o4 call per box (bit for bit: the same
kernels on the same data), and match the oracle (1e-12 normwise).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components
from test_gpu_o4 import usph_box

pytestmark = pytest.mark.gpu


def _boxes(nr, na, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        ext = [int(rng.integers(2, 9)), int(rng.integers(2, 9)), int(rng.integers(2, 9))]
        lo = [int(rng.integers(0, n - e + 1)) for n, e in zip((nr, na, na), ext)]
        hi = [l + e - 1 for l, e in zip(lo, ext)]
        out.append((int(rng.integers(0, 6)), lo, hi, bool(q % 3 == 0)))
    return out


@pytest.mark.parametrize("riemann,gravity", [(2, 0), (1, 1)])
def test_batch_equals_per_box_and_oracle(oracle_lib, riemann, gravity):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200.level import make_box
    po = oracle_lib
    nr, na, g = 16, 16, 5
    kw = dict(nr=nr, na=na, spatial_order=4, riemann_solver=riemann, sun_gravity=gravity)
    shell = hc.Shell(hc.Params(**kw))
    orc = po.OracleLevel(po.make_params(**kw))
    specs = _boxes(nr, na, 12, 7 + riemann)
    works, singles = [], []
    for q, (block, lo, hi, jump) in enumerate(specs):
        u = torch.from_numpy(usph_box(nr, lo, hi, g, seed=q, jump=jump)).cuda()
        v = [hi[d] - lo[d] + 1 for d in range(3)]
        nv = v[0] * v[1] * v[2]
        fsz = [8 * (v[0] + (d == 0)) * (v[1] + (d == 1)) * (v[2] + (d == 2)) for d in range(3)]
        rhs = torch.zeros(8 * nv, dtype=torch.float64, device="cuda")
        flux = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in fsz]
        works.append((make_box(lo, hi, g, block), u, rhs, flux))
        singles.append((make_box(lo, hi, g, block), u, torch.zeros_like(rhs), [torch.zeros_like(f) for f in flux]))
    batch = shell.o4_batch(works, scale=0.5)
    batch.rhs()
    for box, u, rhs, flux in singles:
        if gravity:
            shell.box_gravity_o4(box, u, rhs)
        shell.box_rhs_o4(box, u, rhs, flux, 0.5)
    torch.cuda.synchronize()
    for (box, u, rb, fb), (_, _, rs, fs) in zip(works, singles):
        assert torch.equal(rb, rs)
        for d in range(3):
            assert torch.equal(fb[d], fs[d])
    # two boxes against the oracle
    for q in (0, 5):
        block, lo, hi, jump = specs[q]
        box_o = po.HcBox()
        for d in range(3):
            box_o.lo[d], box_o.hi[d] = lo[d], hi[d]
        box_o.ghost, box_o.block = g, block
        u = works[q][1].cpu().numpy()
        rhs_o = np.zeros(works[q][2].numel())
        if gravity:
            orc.box_gravity_o4(box_o, u, rhs_o)
        orc.box_rhs_o4(box_o, u, rhs_o, None, 0.5)
        err = rel_err_components(works[q][2].cpu().numpy().reshape(8, -1), rhs_o.reshape(8, -1), 0)
        assert err.max() < 1e-12, err
    batch.close()
    shell.close()
