"""Builds libcsdecomp_b200.so for sm_100a with nvcc (csrc/Makefile)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    path = os.path.join(HERE, "libcsdecomp_b200.so")
    if not os.path.exists(path):
        raise RuntimeError("build did not produce libcsdecomp_b200.so")
    return path


if __name__ == "__main__":
    print(build())
