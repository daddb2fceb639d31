"""Readers for the files written by the reference oracle build (oracle/ref).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import glob
import os

import numpy as np

_DTYPES = {("face_owner", 4): np.int32, ("face_neighbour", 4): np.int32, ("face_patch", 4): np.int32,
           ("orthogonal_geometry", 4): np.int32}


def read_records(path):
    """Records written by oracle_driver.cpp writeArray: name, count, width, raw bytes."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        n = int(np.frombuffer(data, np.int64, 1, pos)[0]); pos += 8
        name = data[pos:pos + n].decode(); pos += n
        count, width = (int(v) for v in np.frombuffer(data, np.int64, 2, pos)); pos += 16
        raw = data[pos:pos + count * width]; pos += count * width
        dt = _DTYPES.get((name, width), np.float64)
        arr = np.frombuffer(raw, dt).copy()
        if width in (24,):
            arr = arr.reshape(count, 3)
        out[name] = arr
    return out


def read_system(path):
    """One system_<seq>.bin written by cpu_backend.cpp."""
    with open(path, "rb") as f:
        data = f.read()
    h = np.frombuffer(data, np.int64, 8, 0)
    ncell, nface, comps, lid, lfield, status, iters = (int(v) for v in h[:7])
    pos = 64
    identity = data[pos:pos + lid].decode(); pos += lid
    fieldname = data[pos:pos + lfield].decode(); pos += lfield
    res = np.frombuffer(data, np.float64, 3, pos); pos += 24

    def take(n):
        nonlocal pos
        a = np.frombuffer(data, np.float64, n, pos).copy()
        pos += 8 * n
        return a
    diag, upper, lower = take(ncell), take(nface), take(nface)
    source = take(ncell * comps)
    before = take(ncell * comps)
    after = take(ncell * comps)
    if comps == 3:
        source, before, after = (a.reshape(ncell, 3) for a in (source, before, after))
    return dict(identity=identity, field=fieldname, status=status, iterations=iters, residuals=res,
                diag=diag, upper=upper, lower=lower, source=source, before=before, after=after)


def read_systems(directory):
    return [read_system(p) for p in sorted(glob.glob(os.path.join(directory, "system_*.bin")))]
