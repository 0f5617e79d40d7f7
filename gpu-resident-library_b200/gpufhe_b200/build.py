"""Builds libgpufhe_b200.so in-tree from csrc/ with nvcc for sm_100a.

Every .cu / .cpp under csrc/ is compiled to an object (in parallel, skipped
when up to date) and linked into gpufhe_b200/libgpufhe_b200.so, which the
Python bindings and the C/C++ callers load. Usage: python -m gpufhe_b200.build
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(HERE, "libgpufhe_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOSTCXX,
          f"-I{CSRC}", f"-I{INCLUDE}", "-Xcompiler", "-fvisibility=default"]


def _deps(path: str) -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + [path]


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in _deps(src))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _stale(src, obj):
        return obj
    cmd = [NVCC, *COMMON, *ARCH, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-o", LIB + ".tmp", *objs,
               "-Xlinker", "-Bsymbolic"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    build_driver()
    return LIB


DRIVER_SRC = os.path.join(PKG, "drivers", "plain_chain.cpp")
DRIVER = os.path.join(PKG, "drivers", "_build", "plain_chain")


def build_driver() -> str:
    """drivers/plain_chain: the reference's per-chain EvalMult+Rescale driver
    linked against libgpufhe_b200.so (host code only; rpath to the package)."""
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(DRIVER_SRC),
                                                                 os.path.getmtime(LIB)):
        return DRIVER
    os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
    cmd = [NVCC, "-std=c++17", "-O2", "-ccbin", HOSTCXX, f"-I{INCLUDE}", DRIVER_SRC, "-o", DRIVER + ".tmp",
           f"-L{HERE}", "-lgpufhe_b200", "-Xlinker", "-rpath", "-Xlinker", HERE, "-Wno-deprecated-gpu-targets"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stderr}")
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
