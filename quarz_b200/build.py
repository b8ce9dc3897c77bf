"""Build step of the package: compiles libqz_b200.so for sm_100a (nvcc, in-tree)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> str:
    """Compile quarz_b200/csrc into quarz_b200/libqz_b200.so; returns its path."""
    cmd = ["make", "-j", str(max(1, min(8, os.cpu_count() or 1))), "-C", os.path.join(HERE, "csrc")]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "libqz_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
