"""Build libkcfd.so in-tree with nvcc for sm_100a (B200).

    python -m kcfd.build        (from k-cfd_b200/)  or  kcfd.build.build()

Every .cu / .cpp under k-cfd_b200/csrc is compiled to one shared library next to
this file. Host code is compiled with -ffp-contract=off so the mesh geometry keeps
the reference's rounding; device code keeps FMA contraction.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")
LIB = os.path.join(PKG_DIR, "libkcfd.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, jobs=None):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC, "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [nvcc] + common + ARCH + ["-lineinfo", "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(f"--- {os.path.basename(src)}\n{out}")
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed building libkcfd")
    tmp = LIB + ".tmp"
    link = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("nvcc link failed for libkcfd")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
