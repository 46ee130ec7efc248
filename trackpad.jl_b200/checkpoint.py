"""Checkpoint and resume of long tracks on the host.

A track of many turns can be cut into pieces: ringpass_ over turns
[turn0, turn0 + k), save the state, and later load it and continue with
ringpass_(..., turn=turn0 + k).  Every particle's map sequence depends only on
its own coordinates and the turn numbers (lost particles, lost_flags == 1, are
skipped), so the pieces give the bits of one uninterrupted track.

File format: a JSON header line (format tag, particle count, next turn, a
fingerprint of the lattice's element records, the arrays' byte offsets)
followed by the raw little-endian arrays: coords as N x 6 float64 column-major
(the reference's Matrix layout), lost_flags int64, lost_turn and lost_elem
int32.

  save(path, coords, lost_flags, turn, lat=None, lost_turn=None, lost_elem=None)
  load(path) -> dict(coords, lost_flags, lost_turn, lost_elem, turn, lattice)
  resume_ringpass_(path, lat, beam, nturns, **kw) -> the loaded dict, tracked
"""
import hashlib
import json

import numpy as np

FORMAT = "trackpad-b200-checkpoint-1"


def lattice_fingerprint(lat):
    """SHA-256 of a lattice's packed element records, misalignment rows and
    array fields (None for None)."""
    if lat is None:
        return None
    arr, n, marr, nmis, aux = lat.pack()
    h = hashlib.sha256()
    h.update(f"{n} {nmis}".encode())
    h.update(bytes(arr))
    h.update(bytes(marr))
    h.update(np.ascontiguousarray(aux, dtype=np.float64).tobytes())
    return h.hexdigest()


def save(path, coords, lost_flags, turn, lat=None, lost_turn=None, lost_elem=None):
    """Write the state of a track that continues at turn `turn`."""
    coords = np.asarray(coords)
    if coords.dtype != np.float64 or coords.ndim != 2 or coords.shape[1] != 6:
        raise ValueError("coords must be an (N, 6) float64 array")
    n = coords.shape[0]
    lost = np.ascontiguousarray(lost_flags, dtype=np.int64)
    if lost.shape != (n,):
        raise ValueError("lost_flags must have N entries")
    lt = np.full(n, -1, np.int32) if lost_turn is None else np.ascontiguousarray(lost_turn, dtype=np.int32)
    le = np.full(n, -1, np.int32) if lost_elem is None else np.ascontiguousarray(lost_elem, dtype=np.int32)
    blobs = [np.asfortranarray(coords).tobytes(order="F"), lost.astype("<i8").tobytes(),
             lt.astype("<i4").tobytes(), le.astype("<i4").tobytes()]
    offs, at = [], 0
    for b in blobs:
        offs.append(at)
        at += len(b)
    head = {"format": FORMAT, "n": int(n), "turn": int(turn), "lattice": lattice_fingerprint(lat),
            "offsets": offs, "bytes": at}
    with open(path, "wb") as f:
        f.write((json.dumps(head) + "\n").encode())
        for b in blobs:
            f.write(b)


def load(path):
    """Read a checkpoint: coords (N x 6, column-major), lost_flags, lost_turn,
    lost_elem, the turn to continue at and the lattice fingerprint."""
    with open(path, "rb") as f:
        head = json.loads(f.readline().decode())
        if head.get("format") != FORMAT:
            raise ValueError(f"{path}: not a checkpoint of this library")
        body = f.read()
    if len(body) != head["bytes"]:
        raise ValueError(f"{path}: truncated ({len(body)} of {head['bytes']} bytes)")
    n = head["n"]
    o = head["offsets"]
    coords = np.frombuffer(body, dtype="<f8", count=6 * n, offset=o[0]).reshape((n, 6), order="F").copy(order="F")
    lost = np.frombuffer(body, dtype="<i8", count=n, offset=o[1]).astype(np.int64)
    lt = np.frombuffer(body, dtype="<i4", count=n, offset=o[2]).astype(np.int32)
    le = np.frombuffer(body, dtype="<i4", count=n, offset=o[3]).astype(np.int32)
    return {"coords": coords, "lost_flags": lost, "lost_turn": lt, "lost_elem": le, "turn": head["turn"],
            "lattice": head["lattice"]}


def resume_ringpass_(path, lat, beam, nturns, **kw):
    """Load a checkpoint and continue its track for `nturns` turns from the
    saved turn (the lattice must be the one the checkpoint was written with).
    Keywords go to ringpass_; a time-dependent lattice needs the `time` of the
    saved turn and its `dt_turn`."""
    from . import tracking
    st = load(path)
    fp = lattice_fingerprint(lat)
    if st["lattice"] is not None and fp != st["lattice"]:
        raise ValueError("the checkpoint was written for another lattice")
    tracking.ringpass_(st["coords"], lat, beam, st["lost_flags"], nturns, turn=st["turn"],
                       lost_turn=st["lost_turn"], lost_elem=st["lost_elem"], **kw)
    st["turn"] += int(nturns)
    return st
