"""Checkpoints of a buildup run, and the reference's .npy outputs.

The reference's example loop writes two files every nHistoryOut steps
(example01_basic.py:76-78): ``physicalParticleCount.npy`` (the sum of the
weights at the start of each step so far, as numpy.uint0) and
``particleData.npy`` (the (N, 6) float64 rows [x, y, vx, vy, vz, w] of
getParticleData, particles.pyx:142).  A run restarts from such rows through
setParticleData (particles.pyx:126).  This module writes those files in the
same layout, plus ``macroParticleCount.npy`` and a checkpoint that holds the
device state exactly (the FP32 store as stored, the fixed-point deposit and its
scale, the step counter, the histories, the solver's warm-start state and the
anomaly counters), so a resumed run continues bit for bit.

Format of ``checkpoint.npz``: numpy arrays plus one JSON string ``meta``
(``format``, the run's configuration signature and scalar counters).
"""
import json
import os

import numpy as np

FORMAT = 1
CHECKPOINT = "checkpoint.npz"
PARTICLE_DATA = "particleData.npy"
PHYSICAL_COUNT = "physicalParticleCount.npy"
MACRO_COUNT = "macroParticleCount.npy"

STORE_FIELDS = ("cell", "ox", "oy", "vx", "vy", "vz", "w")
STORE_DTYPES = {"cell": np.int32, "ox": np.float32, "oy": np.float32, "vx": np.float32, "vy": np.float32,
                "vz": np.float32, "w": np.float32}


class CheckpointError(ValueError):
    """A checkpoint that does not belong to the run, or is malformed."""


def write_reference_outputs(directory, particle_rows, physical_count, macro_count):
    """The reference's outputs: (N, 6) float64 rows and the count histories
    (numpy.uint0, the reference's dtype, is numpy.uintp)."""
    os.makedirs(directory, exist_ok=True)
    rows = np.ascontiguousarray(particle_rows, dtype=np.float64).reshape(-1, 6)
    np.save(os.path.join(directory, PARTICLE_DATA), rows)
    np.save(os.path.join(directory, PHYSICAL_COUNT), np.asarray(physical_count, np.float64).astype(np.uintp))
    np.save(os.path.join(directory, MACRO_COUNT), np.asarray(macro_count).astype(np.uintp))


def read_particle_data(path):
    """(N, 6) float64 rows from a particleData.npy (or a directory holding one)."""
    if os.path.isdir(path):
        path = os.path.join(path, PARTICLE_DATA)
    rows = np.load(path, allow_pickle=False)
    if rows.ndim != 2 or rows.shape[1] != 6 or rows.dtype != np.float64:
        raise CheckpointError(f"{path}: expected (N, 6) float64 particle rows, got {rows.shape} {rows.dtype}")
    return rows


def write_checkpoint(directory, signature, store, arrays, counters):
    """store: the FP32 SoA fields (first `count` entries); arrays: other named
    numpy arrays; counters: JSON-able scalars."""
    os.makedirs(directory, exist_ok=True)
    n = None
    out = {}
    for k in STORE_FIELDS:
        a = np.ascontiguousarray(store[k], dtype=STORE_DTYPES[k])
        if n is None:
            n = a.shape[0]
        if a.ndim != 1 or a.shape[0] != n:
            raise CheckpointError(f"store field {k}: {a.shape}, expected ({n},)")
        out["store_" + k] = a
    for k, a in arrays.items():
        if a is not None:
            out["arr_" + k] = np.ascontiguousarray(a)
    meta = {"format": FORMAT, "signature": signature, "count": int(n), "counters": counters}
    out["meta"] = np.array(json.dumps(meta, sort_keys=True))
    tmp = os.path.join(directory, CHECKPOINT + ".tmp.npz")
    np.savez(tmp, **out)
    os.replace(tmp, os.path.join(directory, CHECKPOINT))


def read_checkpoint(directory, signature):
    """(store, arrays, counters) of a checkpoint written for the same run
    configuration; raises CheckpointError otherwise."""
    path = os.path.join(directory, CHECKPOINT) if os.path.isdir(directory) else directory
    with np.load(path, allow_pickle=False) as z:
        try:
            meta = json.loads(str(z["meta"]))
        except KeyError:
            raise CheckpointError(f"{path}: no meta record") from None
        if meta.get("format") != FORMAT:
            raise CheckpointError(f"{path}: format {meta.get('format')}, expected {FORMAT}")
        if meta.get("signature") != signature:
            raise CheckpointError(f"{path}: written for another run configuration: {meta.get('signature')} "
                                  f"!= {signature}")
        n = int(meta["count"])
        store = {}
        for k in STORE_FIELDS:
            a = z["store_" + k]
            if a.dtype != STORE_DTYPES[k] or a.shape != (n,):
                raise CheckpointError(f"{path}: store field {k} is {a.shape} {a.dtype}")
            store[k] = a
        arrays = {k[4:]: z[k] for k in z.files if k.startswith("arr_")}
    return store, arrays, meta["counters"]
