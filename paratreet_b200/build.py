"""Build the CUDA library (sm_100a) in-tree: ``python -m paratreet_b200.build``."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        sys.stderr.write((r.stdout or "") + (r.stderr or ""))
        raise RuntimeError("building libpt_gravity.so failed")
    return os.path.join(HERE, "libpt_gravity.so")


if __name__ == "__main__":
    print(build(verbose=True))
