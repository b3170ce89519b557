"""Build libbempp_b200.so (host C-ABI + sm_100a kernels) in-tree with nvcc.

    python bempp-rs_b200/build.py [--force]

Sources: csrc/host/*.cpp (C++17 host runtime, extern "C" API) and csrc/kernels/*.cu
(CUDA for sm_100a).  Output: bempp-rs_b200/lib/libbempp_b200.so.  Object files go to
bempp-rs_b200/_build/ and are rebuilt only when a source or header is newer.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libbempp_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc()))), "include")


def host_compiler() -> list[str]:
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def headers():
    return glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) + glob.glob(
        os.path.join(CSRC, "**", "*.cuh"), recursive=True) + glob.glob(
        os.path.join(CSRC, "**", "*.inc"), recursive=True) + [
        os.path.join(ROOT, "include", "bempp_b200.h")]


def compile_one(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace(os.sep, "_") + ".o")
    newest_dep = max(os.path.getmtime(p) for p in headers() + [src])
    if force or not os.path.exists(obj) or os.path.getmtime(obj) < newest_dep:
        cmd = [nvcc(), *host_compiler(), *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [host_cxx(), "-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra",
                   f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", f"-I{cuda_include()}",
                   "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")) +
                  glob.glob(os.path.join(CSRC, "kernels", "*.cu")))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, extra), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv))
