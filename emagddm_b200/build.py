"""In-tree build of libemagddm_b200.so (sm_100a) and of the C++ adapter test."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(verbose: bool = False) -> str:
    out = None if verbose else subprocess.DEVNULL
    subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc")], stdout=out)
    return os.path.join(HERE, "libemagddm_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
