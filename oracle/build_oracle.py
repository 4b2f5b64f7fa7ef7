"""Build the CPU oracle shared library (test infrastructure only).

``python oracle/build_oracle.py`` compiles ``oracle/gmf_oracle.c`` into
``oracle/libgmf_oracle.so`` with strict IEEE semantics (no FMA contraction, no
fast-math), so its float32 / float64 arithmetic matches numpy and torch CPU
operation for operation.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "gmf_oracle.c")
LIB = os.path.join(HERE, "libgmf_oracle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = [
        "gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-fPIC", "-shared",
        "-ffp-contract=off", "-fno-fast-math", "-fexcess-precision=standard",
        "-o", LIB, SRC, "-lpthread", "-lm",
    ]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
