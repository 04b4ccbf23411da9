"""Raw-binary level checkpoints (heliocubed_b200.checkpoint): round trip is
bit-exact with options, model time, step and attributes; corrupted, truncated
or foreign files are rejected; a failed write leaves the old file intact."""
from __future__ import annotations

import os

import numpy as np
import pytest

from heliocubed_b200 import checkpoint
from heliocubed_b200.level import Params


def _state(p, seed=0):
    return np.random.default_rng(seed).standard_normal(6 * 8 * p.nr * p.na * p.na)


def test_round_trip_bit_exact(tmp_path):
    p = Params(nr=6, na=5, spatial_order=4, riemann_solver=2)
    s = _state(p)
    path = str(tmp_path / "lvl.hcb")
    checkpoint.save(path, p, s, 1234.5, step=17, attributes={"cme_inserted_count": 2})
    q, t, time, step, attrs = checkpoint.load(path)
    assert q == p and time == 1234.5 and step == 17 and attrs == {"cme_inserted_count": 2}
    assert np.array_equal(t, s)


def test_rejects_bad_files(tmp_path):
    p = Params(nr=4, na=4)
    path = str(tmp_path / "a.hcb")
    checkpoint.save(path, p, _state(p), 0.0)
    raw = open(path, "rb").read()
    bad = str(tmp_path / "b.hcb")
    open(bad, "wb").write(b"NOTACKPT" + raw[8:])
    with pytest.raises(checkpoint.CheckpointError):
        checkpoint.load(bad)
    open(bad, "wb").write(raw[:-8])
    with pytest.raises(checkpoint.CheckpointError):
        checkpoint.load(bad)
    flipped = bytearray(raw)
    flipped[-3] ^= 0x40
    open(bad, "wb").write(bytes(flipped))
    with pytest.raises(checkpoint.CheckpointError):
        checkpoint.load(bad)


def test_wrong_size_state_is_refused_and_old_file_kept(tmp_path):
    p = Params(nr=4, na=4)
    path = str(tmp_path / "c.hcb")
    s = _state(p)
    checkpoint.save(path, p, s, 1.0)
    with pytest.raises(checkpoint.CheckpointError):
        checkpoint.save(path, p, s[:-1], 2.0)
    assert checkpoint.load(path)[2] == 1.0
    assert not [f for f in os.listdir(tmp_path) if ".tmp." in f]
