"""Build recipe of the in-tree CUDA library (sm_100a only).

    python -m z2_gauge_zfy_b200.build

compiles ``csrc/z2_api.cu`` into ``libz2dqmc.so`` next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "z2_api.cu")
OUT = os.path.join(HERE, "libz2dqmc.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
              "-std=c++17", "-shared", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))
            if f.endswith((".cu", ".cuh", ".h"))] + \
        [os.path.join(os.path.dirname(HERE), "include", "z2dqmc.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


DRIVER_SRC = os.path.join(HERE, "csrc", "z2_main.cpp")
DRIVER = os.path.join(HERE, "z2_gauge_b200")


def build_driver(force: bool = False) -> str:
    """The host driver (restates src/main.f90 over the C ABI), linked to the
    in-tree library with an $ORIGIN rpath."""
    if (not force and os.path.exists(DRIVER)
            and os.path.getmtime(DRIVER) >= max(os.path.getmtime(DRIVER_SRC),
                                                os.path.getmtime(OUT))):
        return DRIVER
    tmp = f"{DRIVER}.tmp.{os.getpid()}"
    cmd = ["g++", "-O2", "-std=c++17", DRIVER_SRC, "-L" + HERE, "-lz2dqmc",
           "-Wl,-rpath,$ORIGIN", "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, DRIVER)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        # per-process temporary name: ranks that start together on a fresh
        # checkout may build side by side; os.replace makes the swap atomic
        tmp = f"{OUT}.tmp.{os.getpid()}"
        cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, SRC]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, OUT)
    build_driver(force)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
