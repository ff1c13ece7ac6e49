"""Build recipe for libselm_b200.so (nvcc, sm_100a only) and the selm_b200 CLI."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "lib", "libselm_b200.so")


if __name__ == "__main__":
    print(build())
