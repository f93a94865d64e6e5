"""Build the B200 library (libbeep_b200.so) and the `beep` CLI in-tree with nvcc
for sm_100a. Objects go to beep_b200/_build/ (git-ignored); the shared
library and CLI land next to this file so they travel with the repository."""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbeep_b200.so")
CLI = os.path.join(HERE, "beep")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
# The system g++ ships libgomp; a compiler named by CC/CXX may not.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-ccbin", HOST_CXX, "-I", INCLUDE,
          "-Xcompiler", "-fPIC,-fopenmp,-Wall", "-Wno-deprecated-declarations"]

LIB_SOURCES = ["graph.cu", "count.cu", "plan.cpp", "io.cpp", "convert.cpp", "api.cpp", "serve.cpp"]
HEADERS = ["internal.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    deps = [path, os.path.join(INCLUDE, "beep.h")] + [os.path.join(CSRC, h) for h in HEADERS]
    if _newer(obj, deps):
        cmd = [NVCC, *COMMON, *ARCH, "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, *COMMON, "-x", "c++", "-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(_compile, LIB_SOURCES))
    if _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"]
        subprocess.run(cmd, check=True, capture_output=not verbose)
    cli_obj = _compile("cli.cpp")
    if _newer(CLI, [cli_obj, LIB]):
        cmd = [NVCC, *ARCH, "-ccbin", HOST_CXX, "-o", CLI, cli_obj, "-L", HERE, "-lbeep_b200",
               "-Xlinker", "-rpath,$ORIGIN", "-Xcompiler", "-fopenmp", "-lgomp"]
        subprocess.run(cmd, check=True, capture_output=not verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
