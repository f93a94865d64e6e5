"""Compile the reference implementation itself for sm_100a as a second oracle.

TEST INFRASTRUCTURE ONLY. Compiles the reference's single translation unit
src/main.cu where it lies (read-only, never copied) with the reference
Makefile's CUDA flags, with the nauty stand-in in oracle/ref_shim on the
include path (nauty is not vendored by the reference). The binary goes to
oracle/_ref/beep_ref (git-ignored; it travels to GPU machines with the
working tree). Nothing here runs on a machine without the reference sources.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: BEEP_REFERENCE_ROOT, else a directory named
# "reference" beside this repository's root.
REF_ROOT = os.environ.get("BEEP_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT_DIR = os.path.join(HERE, "_ref")
BINARY = os.path.join(OUT_DIR, "beep_ref")


def available() -> bool:
    return os.path.exists(os.path.join(REF_ROOT, "src", "main.cu"))


def build(force: bool = False) -> str:
    src = os.path.join(REF_ROOT, "src", "main.cu")
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    if os.path.exists(BINARY) and not force:
        return BINARY
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    host = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    # '#include "../nauty/nauty.h"' in subgraph_matching.cuh resolves against
    # each -I directory D as D/../nauty/nauty.h -> oracle/ref_shim/nauty/nauty.h
    inc = os.path.join(HERE, "ref_shim", "inc")
    cmd = [nvcc, "-ccbin", host, "-g", "-w", "-Xcompiler", "-fopenmp", "-lineinfo", "-O3", "-DCUDA", "-DNOT_IMPL",
           "-arch=sm_100a", "-gencode=arch=compute_100a,code=sm_100a", "-I", inc, src, "-o", BINARY,
           "-lcuda", "-lgomp"]
    subprocess.run(cmd, check=True)
    return BINARY


def build_if_available() -> str | None:
    if not available():
        return None
    try:
        return build()
    except (subprocess.CalledProcessError, OSError) as e:  # recorded, not fatal: the port oracle remains
        print(f"reference build failed: {e}")
        return None


if __name__ == "__main__":
    print(build(force=True))
