"""DCD trajectory output (CPU: the writer needs no GPU when given host positions).

The layout is pinned by the reference's own recorded trajectory: the first
frames of data/cases/SELM/DIffusion Coefficient/1base.dcd (written by LAMMPS'
dump dcd; cut by tests/golden/make_dcd_fixture.py) read back with the
header the paper case implies, and a file written by selm_dcd_* has the same
record structure and reads back exactly (positions as float32)."""
import ctypes as C
import os

import numpy as np

from monomers2026_b200 import _lib
from monomers2026_b200.dcd import read_dcd

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "dcd_1base_head.dcd")


def test_reference_trajectory_header_and_frames():
    d = read_dcd(FIX)
    # 2e7 steps dumped every 4000 from step 0, four atoms, timestep 0.005, 6-unit periodic cell
    assert (d["nset"], d["istart"], d["nsavc"], d["nstep"]) == (5001, 0, 4000, 20000000)
    assert abs(d["dt"] - 0.005) < 1e-7 and d["natoms"] == 4 and d["has_cell"]
    assert d["titles"][0].startswith("Written by LAMMPS")
    assert d["xyz"].shape == (3, 4, 3)
    assert np.allclose(d["cells"][0], [6.0, 0.0, 6.0, 0.0, 0.0, 6.0])


def _write(path, x_frames, dt=0.005, first=0, interval=4000, box=6.0):
    L = _lib.load()
    h = C.c_void_p()
    b = (C.c_double * 3)(box, box, box)
    assert L.selm_dcd_open(path.encode(), x_frames.shape[1], dt, first, interval, b, C.byref(h)) == 0
    for x in x_frames:
        xx = np.ascontiguousarray(x, np.float64)
        assert L.selm_dcd_write(h, xx.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert L.selm_dcd_close(h) == 0


def test_written_trajectory_reads_back(tmp_path):
    rng = np.random.default_rng(3)
    frames = rng.uniform(-3, 3, (5, 4, 3))
    p = str(tmp_path / "t.dcd")
    _write(p, frames)
    d = read_dcd(p)
    assert (d["nset"], d["istart"], d["nsavc"], d["nstep"]) == (5, 0, 4000, 16000)
    assert abs(d["dt"] - 0.005) < 1e-7 and d["natoms"] == 4
    assert np.array_equal(d["xyz"], frames.astype(np.float32))
    assert np.allclose(d["cells"], [6.0, 0.0, 6.0, 0.0, 0.0, 6.0])


def test_layout_matches_the_reference_file(tmp_path):
    ref = open(FIX, "rb").read()
    frames = read_dcd(FIX)["xyz"].astype(np.float64)
    p = str(tmp_path / "same.dcd")
    _write(p, frames)
    ours = open(p, "rb").read()
    assert len(ours) == len(ref)
    # header apart from the frame count and last step (8..12, 20..24), titles apart,
    # then atom count and frames: byte for byte
    assert ours[:8] == ref[:8] and ours[12:20] == ref[12:20] and ours[24:92] == ref[24:92]
    assert ours[92 + 172:] == ref[92 + 172:]
