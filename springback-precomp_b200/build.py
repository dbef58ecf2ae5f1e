"""Builds the CUDA library of the package, in tree: libsbk.so beside this file.

nvcc cross-compiles for sm_100a (B200) without a GPU. The library exports
the C ABI of include/sbk.h and nothing else; it links the CUDA runtime
statically, so it loads on any box with the driver, and cuSOLVER and
cuSPARSE (the free-free block's factorisation) dynamically, by soname.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsbk.so")
SOURCES = ["sbk_element.cu", "sbk_assembly.cu", "sbk_contact.cu", "sbk_capi.cu", "sbk_schedule.cu", "sbk_noalloc.cu",
           "sbk_pattern.cu", "sbk_return.cu",
           "sbk_partition.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(verbose_ptxas: bool = False):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "sbk.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + flags(verbose_ptxas) + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose_ptxas or p.returncode != 0:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
    tmp = LIB + ".tmp"
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "lib64")
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static", "-L" + cuda_lib,
                                                                      "-lcusolver", "-lcusparse"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
