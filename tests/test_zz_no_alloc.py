"""hc_level_rk4_step_noalloc: the RK4 level step for callers that cannot
allocate device memory while they step (stream capture, a host framework
that owns all device memory, a serving loop that must not wait on the
allocator).  Its stage workspace is a fixed array inside the library.

Called through the C ABI and checked against hc_level_rk4_step, the
allocating entry point, on two calls in a row, with the tolerance of the
other operator tests (1e-12 normwise per component), after a call on a level
of another shape has left its data in the shared array.  The file sorts last so
a run that stops at the first failure has run every other test before it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available, rel_err_components

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def test_noalloc_step_matches_allocating_step():
    _need_gpu()
    import torch

    import heliocubed_b200 as hc
    lib = hc.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # A first call on a level of another shape leaves its (non-zero) stage
    # data in the shared array at offsets the 12 x 10 level uses
    # differently: the steps below must not read any of it.
    other = hc.Shell(hc.Params(nr=20, na=18, limiter=3, riemann_solver=1))
    ju_other = other.init(hc.InitSpec.seeded(3, 20, 18, margin=2))
    dt_other = 0.4 / other.inv_dt_max(ju_other).item()
    rc = lib.hc_level_rk4_step_noalloc(other._ctx, C.c_void_p(ju_other.data_ptr()), dt_other, 0.0, stream)
    assert rc == 0, lib.hc_last_error()
    torch.cuda.synchronize()
    assert other.valid(ju_other)
    other.close()

    nr, na = 12, 10
    shell = hc.Shell(hc.Params(nr=nr, na=na, limiter=3, riemann_solver=2, sun_gravity=1))
    ju = shell.init(hc.InitSpec.seeded(7, nr, na, margin=2))
    a = ju.clone()
    b = ju.clone()
    dt = 0.4 / shell.inv_dt_max(ju).item()
    for call in range(2):
        t = call * dt
        shell.rk4_step(a, dt, t)
        rc = lib.hc_level_rk4_step_noalloc(shell._ctx, C.c_void_p(b.data_ptr()), dt, t, stream)
        assert rc == 0, lib.hc_last_error()
        torch.cuda.synchronize()
        err = rel_err_components(b.cpu().numpy().reshape(6, 8, -1), a.cpu().numpy().reshape(6, 8, -1))
        assert err.max() <= 1e-12, (call, err)
    assert shell.valid(b)
    shell.close()


def test_noalloc_step_rejects_levels_beyond_its_workspace():
    _need_gpu()
    import torch

    import heliocubed_b200 as hc
    shell = hc.Shell(hc.Params(nr=24, na=24))
    ju = shell.new_state()
    lib = hc.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.hc_level_rk4_step_noalloc(shell._ctx, C.c_void_p(ju.data_ptr()), 1.0, 0.0, stream)
    assert rc == -1  # HC_ERR_ARG, before any launch
    msg = lib.hc_last_error().decode()
    assert "needs" in msg and "2097152" in msg, msg
    shell.close()
