"""A device-resident solve resumes bit-identically from a checkpoint (the
reference's Write_Checkpoint / ReadCheckpointState cycle,
src/MHD_IO.H:1390-1465): a served cone-CME request, admitted on the device
with its insertion schedule, advances 3 RK4 steps (device CFL dt), is
written with heliocubed_b200.checkpoint, advances 3 more; a fresh context
loads the checkpoint, sets the request's insertion schedule again and
advances the same 3 steps.  Both end states and model times must be equal
bit for bit, at either order.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [2, 4])
def test_device_solve_resumes_bit_identically(tmp_path, order):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    import heliocubed_b200 as hc
    from heliocubed_b200 import checkpoint, serve

    cone = serve.Cone(speed_kms=1200.0, half_width_deg=30.0, lat_deg=10.0, lon_deg=-20.0, density_ratio=4.0)
    req = serve.Request(0, 16, 16, order, 0, cone=cone)
    params = dataclasses.replace(req.params(), autotune=0)
    sh = hc.Shell(params)
    ju = sh.new_state()
    t = torch.zeros(1, dtype=torch.float64, device="cuda")
    serve.admit(sh, req, ju, t)
    sh.advance(ju, 3, t)
    torch.cuda.synchronize()
    path = str(tmp_path / "solve.hcb")
    checkpoint.save(path, params, ju, float(t.item()), step=3,
                    attributes={"cone": dataclasses.asdict(cone), "order": order})
    sh.advance(ju, 3, t)
    torch.cuda.synchronize()
    uninterrupted, t_end = ju.cpu().numpy(), float(t.item())
    sh.close()

    p, state, time, step, attrs = checkpoint.load(path)
    assert p == params and step == 3 and attrs["order"] == order
    sh2 = hc.Shell(p)
    ju2 = torch.from_numpy(state).cuda()
    t2 = torch.tensor([time], dtype=torch.float64, device="cuda")
    sh2.set_cme_schedule([serve.Cone(**attrs["cone"]).prepared(p)])
    sh2.advance(ju2, 3, t2)
    torch.cuda.synchronize()
    assert float(t2.item()) == t_end
    assert np.array_equal(ju2.cpu().numpy(), uninterrupted)
    assert sh2.valid(ju2)
    sh2.close()
