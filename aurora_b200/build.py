"""Builds the sm_100a shared library in-tree (nvcc via make): aurora_b200/lib/libaurora_b200.so."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, verbose: bool = False) -> str:
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building libaurora_b200.so failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stdout)
    return os.path.join(HERE, "lib", "libaurora_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
