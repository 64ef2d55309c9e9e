"""Build recipe of the C restatement (oracle/c/z2cpu.c -> oracle/libz2cpu.so),
linked to the reference-LAPACK routines of SciPy's bundled OpenBLAS.
Test infrastructure and CPU baseline only.

    python -m oracle.build_cpu
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "z2cpu.c")
OUT = os.path.join(HERE, "libz2cpu.so")


def openblas():
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    libs = glob.glob(os.path.join(libdir, "libscipy_openblas*.so"))
    if not libs:
        raise RuntimeError("SciPy's bundled OpenBLAS not found")
    return libdir, os.path.basename(libs[0])


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    libdir, lib = openblas()
    # a per-process temporary name: ranks started together on a fresh
    # checkout build side by side and the last os.replace wins
    tmp = f"{OUT}.tmp.{os.getpid()}"
    cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", SRC, "-o", tmp,
           "-L" + libdir, "-l:" + lib, "-Wl,-rpath," + libdir, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
