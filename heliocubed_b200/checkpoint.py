"""Level checkpoints in a raw binary format.

The reference writes its checkpoints as HDF5 (MBLevelBoxData through
Proto's HDF5Handler::writeMBLevel, with the CME insertion count as a level
attribute, src/MHD_IO.H:1322-1465).  HDF5 is not available here, so a
checkpoint is one file holding

    8 bytes   magic b"HCB200CK"
    8 bytes   little-endian uint64: length L of the JSON header
    L bytes   JSON header: format version, hc_params fields, layout, model
              time, step count, extra attributes (e.g. cme_inserted_count),
              and the SHA-256 of the payload
    payload   the level state JU, float64 little-endian, in the layout of
              hc_level_state_size: [panel 6][component 8][k na][j na][i nr]

Writes go to a temporary file in the same directory, are flushed to disk and
renamed over the target, so a crash never leaves a truncated checkpoint
under the target name.  Reads verify magic, sizes and the payload hash.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
import struct

import numpy as np

MAGIC = b"HCB200CK"
VERSION = 1


class CheckpointError(RuntimeError):
    pass


def _as_numpy(state) -> np.ndarray:
    if hasattr(state, "detach"):  # torch tensor, on any device
        state = state.detach().cpu().numpy()
    a = np.ascontiguousarray(np.asarray(state, dtype="<f8"))
    return a.reshape(-1)


def save(path: str, params, state, time: float, step: int = 0, attributes: dict | None = None) -> None:
    """Write `state` (numpy array or torch tensor with 6*8*nr*na*na
    doubles) of a level with options `params` (heliocubed_b200.Params)."""
    a = _as_numpy(state)
    expect = 6 * 8 * params.nr * params.na * params.na
    if a.size != expect:
        raise CheckpointError(f"state has {a.size} doubles, the {params.nr}x{params.na}^2x6 level needs {expect}")
    payload = a.tobytes()
    header = {
        "version": VERSION,
        "params": dataclasses.asdict(params),
        "layout": "JU[6][8][na][na][nr] float64 little-endian, radial index fastest",
        "time": float(time),
        "step": int(step),
        "attributes": dict(attributes or {}),
        "payload_bytes": len(payload),
        "sha256": hashlib.sha256(payload).hexdigest(),
    }
    hb = json.dumps(header, sort_keys=True).encode()
    tmp = f"{path}.tmp.{os.getpid()}"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(hb)))
        f.write(hb)
        f.write(payload)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)
    # make the rename itself durable: sync the directory entry
    try:
        fd = os.open(os.path.dirname(os.path.abspath(path)), os.O_RDONLY)
    except OSError:
        return  # platforms where a directory cannot be opened
    try:
        os.fsync(fd)
    except OSError:
        pass
    finally:
        os.close(fd)


def load(path: str):
    """Read a checkpoint: (Params, state as a float64 numpy array, time,
    step, attributes)."""
    from .level import Params
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise CheckpointError(f"{path}: not a checkpoint (bad magic)")
        raw = f.read(8)
        if len(raw) != 8:
            raise CheckpointError(f"{path}: truncated header")
        (n,) = struct.unpack("<Q", raw)
        hb = f.read(n)
        if len(hb) != n:
            raise CheckpointError(f"{path}: truncated header")
        header = json.loads(hb)
        if header.get("version") != VERSION:
            raise CheckpointError(f"{path}: unsupported version {header.get('version')}")
        payload = f.read()
    if len(payload) != header["payload_bytes"]:
        raise CheckpointError(f"{path}: payload has {len(payload)} bytes, expected {header['payload_bytes']}")
    if hashlib.sha256(payload).hexdigest() != header["sha256"]:
        raise CheckpointError(f"{path}: payload hash mismatch")
    params = Params(**header["params"])
    state = np.frombuffer(payload, dtype="<f8").copy()
    return params, state, header["time"], header["step"], header["attributes"]
