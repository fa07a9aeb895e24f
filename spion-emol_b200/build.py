"""Build libscatt_b200.so (sm_100a) in-tree with nvcc, and the C++ host driver.

    python spion-emol_b200/build.py [--force] [-j N]

Objects go to spion-emol_b200/_build/; the shared library lands next to this
file so it travels with the source tree.  host/scan_driver (the command-line
use of host/scatt_b200.hpp) links against it with an $ORIGIN-relative rpath.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libscatt_b200.so")
INCLUDE = os.path.join(ROOT, "include")
HOST = os.path.join(HERE, "host")
DRIVER = os.path.join(HOST, "scan_driver")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(os.path.join(CSRC, f))
    return out


def headers_mtime():
    m = 0.0
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def compile_one(src, force, hm, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        om = os.path.getmtime(obj)
        if om >= os.path.getmtime(src) and om >= hm:
            return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, *COMMON, "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj]
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-Wall", "-I", INCLUDE, "-I", CSRC,
               "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj, None


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hm = headers_mtime()
    srcs = sources()
    objs = []
    errs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, err in ex.map(lambda s: compile_one(s, force, hm, verbose), srcs):
            objs.append(obj)
            if err:
                errs.append(err)
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_host(force)
    return LIB


def build_host(force: bool = False) -> str:
    """g++ build of host/scan_driver against the in-tree library."""
    src = os.path.join(HOST, "scan_driver.cpp")
    deps = [src, os.path.join(HOST, "scatt_b200.hpp"), os.path.join(INCLUDE, "scatt_b200.h"), LIB]
    if not force and os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(d) for d in deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-I", HOST, src, "-o", DRIVER,
           "-L", HERE, "-lscatt_b200", "-Wl,-rpath,$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host driver build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return DRIVER


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true", help="print ptxas resource usage")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
