"""Builds the sm_100a library (parallax_b200/libpxs.so) with nvcc and make.

`python -m parallax_b200.build` or build(); the checker libraries under
oracle/ are built separately by __graft_entry__.build().
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"], check=True)
    return os.path.join(HERE, "libpxs.so")


if __name__ == "__main__":
    print(build())
