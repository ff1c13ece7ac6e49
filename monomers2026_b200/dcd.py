"""Reading DCD trajectories (the layout LAMMPS' "dump ... dcd" writes, and
selm_dcd_* / the selm_b200 executable write): header, titles, atom count,
then per frame an optional unit cell and X, Y, Z as float32 records."""
from __future__ import annotations

import struct

import numpy as np


def _records(buf: bytes):
    o = 0
    while o + 4 <= len(buf):
        n = struct.unpack_from("<i", buf, o)[0]
        if o + 8 + n > len(buf):
            return
        if struct.unpack_from("<i", buf, o + 4 + n)[0] != n:
            raise ValueError("DCD record lengths do not match")
        yield buf[o + 4:o + 4 + n]
        o += 8 + n


def read_dcd(path: str) -> dict:
    """{'nset', 'istart', 'nsavc', 'nstep', 'dt', 'has_cell', 'titles', 'natoms',
    'cells' [F, 6], 'xyz' [F, natoms, 3]} for the frames present in the file."""
    buf = open(path, "rb").read()
    recs = _records(buf)
    h = next(recs)
    if len(h) != 84 or h[:4] != b"CORD":
        raise ValueError("not a DCD file")
    ic = struct.unpack("<20i", h[4:84])
    dt = struct.unpack("<f", h[40:44])[0]
    t = next(recs)
    nt = struct.unpack_from("<i", t)[0]
    titles = [t[4 + 80 * i:4 + 80 * (i + 1)].rstrip(b"\0 ").decode(errors="replace") for i in range(nt)]
    natoms = struct.unpack("<i", next(recs))[0]
    has_cell = ic[10] == 1
    cells, xyz = [], []
    rest = list(recs)
    per = 4 if has_cell else 3
    for k in range(len(rest) // per):
        r = rest[k * per:(k + 1) * per]
        if has_cell:
            cells.append(struct.unpack("<6d", r[0]))
            r = r[1:]
        xyz.append(np.stack([np.frombuffer(q, "<f4") for q in r], axis=1))
    return {"nset": ic[0], "istart": ic[1], "nsavc": ic[2], "nstep": ic[3], "dt": dt, "has_cell": has_cell,
            "titles": titles, "natoms": natoms, "cells": np.array(cells), "xyz": np.array(xyz)}
