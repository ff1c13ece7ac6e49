"""Cut the first frames of the reference's recorded trajectory
(data/cases/SELM/DIffusion Coefficient/1base.dcd, written by LAMMPS' dump dcd)
into a small fixture that pins the DCD layout: header, titles and atom count
(276 bytes) plus three frames of 128 bytes each."""
import os
import sys

SRC = os.path.join(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SELM_REFERENCE_ROOT", "/root/reference"),
                   "data", "cases", "SELM", "DIffusion Coefficient", "1base.dcd")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dcd_1base_head.dcd")
buf = open(SRC, "rb").read()
open(OUT, "wb").write(buf[:276 + 3 * 128])
print("wrote", OUT, 276 + 3 * 128, "bytes")
