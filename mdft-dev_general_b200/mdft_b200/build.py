"""Compile the CUDA engine (sm_100a) in-tree: csrc/ -> mdft_b200/libmdft_b200.so."""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(PKG), "csrc")
SO = os.path.join(PKG, "libmdft_b200.so")


def build(force: bool = False, verbose: bool = False) -> str:
    cmd = ["make", "-C", CSRC]
    if force:
        cmd.append("-B")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        sys.stderr.write(out.stdout + out.stderr)
        raise RuntimeError("building libmdft_b200.so failed")
    if verbose:
        sys.stdout.write(out.stdout)
    return SO


if __name__ == "__main__":
    print(build(force="-B" in sys.argv, verbose=True))
