"""The stage-tile autotuner's host side without a GPU: the candidate tiles
(hc_stage_tiles) are 128-thread cell tiles with register caps that fit the
SM, and the option travels through hc_params."""
from __future__ import annotations

import ctypes as C

import numpy as np

import heliocubed_b200 as hc
from heliocubed_b200 import _native as N
from heliocubed_b200.level import stage_tiles


def test_tiles_are_valid_cta_shapes():
    t = stage_tiles()
    assert t.shape[0] >= 4 and t.shape[1] == 5
    assert (t[:, 0] * t[:, 1] * t[:, 2] == 128).all()
    # the default tile (16 x 4 x 2) comes first
    assert tuple(t[0, :3]) == (16, 4, 2)
    # shapes or register caps differ between candidates
    assert len({tuple(r) for r in t}) == t.shape[0]
    # register caps: 65536 registers per SM over the resident threads
    for x, y, z, mb_rus, mb_roe in t:
        for mb in (mb_rus, mb_roe):
            assert 1 <= mb and 65536 // (mb * 128) >= 64


def test_autotune_option_in_params():
    p = hc.Params(nr=8, na=8, autotune=1).to_c()
    assert p.autotune == 1
    assert C.sizeof(N.HcParams) == 4 * 16 + 8 * 14


def test_capacity_is_respected():
    lib = N.lib()
    buf = (C.c_int * 6)(*([-7] * 6))
    n = lib.hc_stage_tiles(buf, 1)
    assert n == stage_tiles().shape[0]
    assert buf[5] == -7 and buf[0] == 16


def test_o4_variants_table():
    from heliocubed_b200.level import o4_variants
    v = o4_variants()
    assert v.shape == (3, 3)
    # variant 0 is the default register cap of each kernel; all caps fit 128-thread CTAs
    assert tuple(v[:, 0]) == (6, 4, 3)
    assert (v >= 1).all() and (65536 // (v * 128) >= 64).all()
