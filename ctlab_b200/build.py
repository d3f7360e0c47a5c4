"""Builds libctlab_b200.so in-tree for sm_100a (``python -m ctlab_b200.build``)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    csrc = os.path.join(HERE, "csrc")
    r = subprocess.run(["make", "-C", csrc, f"-j{jobs}"], capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError("building libctlab_b200.so failed")
    return os.path.join(HERE, "libctlab_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
