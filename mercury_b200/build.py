"""In-tree build of the sm_100a library and the drop-in programs.

``build()`` runs the Makefile in mercury_b200/csrc (nvcc
-gencode arch=compute_100a,code=sm_100a -lineinfo for every .cu file), which
writes mercury_b200/lib/libmercury_b200.so and mercury_b200/bin/{tc_challenge,sm}.
nvcc cross-compiles, so this works on a machine without a GPU.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int = 8, verbose: bool = False) -> None:
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    if not verbose:
        cmd.append("-s")
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(verbose=True)
