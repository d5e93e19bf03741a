"""Input-bundle reader and writer (the format of warp-fdtd's results/warp_reference/<case>/).

A bundle is a directory with `inputs.npz` (arrays) and `manifest.json`
(objects, dt, steps, settings, SHA-256 of inputs.npz).  The reader follows
warp_fdtd/solver.py:60-66 (checksum check, eager load); the writer produces the
same keys and manifest fields the FDTDX exporter writes
(baseline/export_case.py:76-190) for the objects this solver consumes, so a
bundle written here also loads in the reference Solver.
"""

import hashlib
import io
import json
from pathlib import Path

import numpy as np


def read_bundle(case):
    path = Path(case)
    meta = json.loads((path / "manifest.json").read_text())
    raw = path / "inputs.npz"
    blob = raw.read_bytes()
    if hashlib.sha256(blob).hexdigest() != meta["inputs_sha256"]:
        raise ValueError("Input bundle checksum mismatch")
    with np.load(io.BytesIO(blob)) as data:
        arrays = {n: data[n] for n in data.files}
    return meta, arrays


def write_bundle(path, arrays, meta):
    """Write inputs.npz + manifest.json; fills inputs_sha256 and the array table."""
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    buf = io.BytesIO()
    np.savez(buf, **arrays)
    blob = buf.getvalue()
    (path / "inputs.npz").write_bytes(blob)
    meta = dict(meta)
    meta["inputs_sha256"] = hashlib.sha256(blob).hexdigest()
    meta["arrays"] = {
        k: {"shape": list(np.shape(v)), "dtype": str(np.asarray(v).dtype)}
        for k, v in arrays.items()
    }
    (path / "manifest.json").write_text(json.dumps(meta, indent=1) + "\n")
    return path
