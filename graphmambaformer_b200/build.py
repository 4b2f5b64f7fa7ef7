"""Build the CUDA library ``graphmambaformer_b200/lib/libgmf_align.so``.

The library is compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) straight from ``csrc/*.cu`` with nvcc; it
links nothing but the CUDA runtime and exposes the C ABI of
``include/gmf_align.h``.  ``python -m graphmambaformer_b200.build`` rebuilds it.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libgmf_align.so")
PROBE_SRC = os.path.join(CSRC, "probe", "int_probe.cu")
PROBE_LIB = os.path.join(LIBDIR, "libgmf_probe.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the gmf CUDA library cannot be built")
    return path


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build_probe(force: bool = False) -> str:
    """The integer-ALU throughput probe used as the SW roofline denominator."""
    if not force and os.path.exists(PROBE_LIB) and os.path.getmtime(PROBE_LIB) >= os.path.getmtime(PROBE_SRC):
        return PROBE_LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = PROBE_LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-cudart",
                    "static", "-o", tmp, PROBE_SRC], check=True)
    os.replace(tmp, PROBE_LIB)
    return PROBE_LIB


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    build_probe(force)
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj, *(extra or [])]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    # the CUDA runtime is linked statically: the library then works next to any
    # other runtime in the process (torch's, or none) and needs no library path
    subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
