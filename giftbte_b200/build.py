"""Builds the in-tree shared library giftbte_b200/_build/libgiftbte_b200.so
(and the giftbte_cli drop-in executable) for sm_100a with nvcc.

    python -m giftbte_b200.build [--force]

Host sources are compiled by nvcc's host compiler; the CUDA translation unit
targets compute_100a/sm_100a only. The CUDA runtime is linked statically so
the library loads on any machine with the NVIDIA driver.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libgiftbte_b200.so")
CLI = os.path.join(OUT, "giftbte_cli")

SOURCES = ["deck.cpp", "mesh.cpp", "angles.cpp", "capi.cpp", "solver.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _digest() -> str:
    h = hashlib.sha256()
    for dirpath, _, files in sorted(os.walk(CSRC)):
        for name in sorted(files):
            with open(os.path.join(dirpath, name), "rb") as f:
                h.update(name.encode() + f.read())
    with open(os.path.join(ROOT, "include", "giftbte.h"), "rb") as f:
        h.update(f.read())
    h.update(" ".join(ARCH).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    stamp = os.path.join(OUT, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(CLI) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    cc = nvcc()
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include")]
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OUT, s + ".o")
        cmd = [cc] + ARCH + common + ["-c", src, "-o", obj]
        if s.endswith(".cu"):
            cmd += ["-Xptxas", "-O3"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(obj)
    subprocess.check_call([cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    cli_obj = os.path.join(OUT, "cli.cpp.o")
    subprocess.check_call([cc] + ARCH + common + ["-c", os.path.join(CSRC, "cli", "cli.cpp"), "-o", cli_obj])
    subprocess.check_call([cc] + ARCH + ["-o", CLI, cli_obj, "-L", OUT, "-lgiftbte_b200",
                                         "-Xlinker", "-rpath,$ORIGIN"])
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
