"""Builds libontc.so in-tree (openntc_b200/libontc.so) with nvcc for sm_100a.

Usage:  python -m openntc_b200.build [--force] [--verbose]

Every .cu/.cpp under openntc_b200/csrc is compiled once (object files are cached under
openntc_b200/_build, keyed by source and header modification times) and linked into one
shared library that exports the C ABI declared in include/ontc.h.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libontc.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = CUDA / "bin" / "nvcc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++20", "-I", str(ROOT / "include"), "-I", str(CSRC)]
NVCC_FLAGS = ARCH + COMMON + ["-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
                              "--expt-relaxed-constexpr"]
CXX_FLAGS = COMMON + ["-fPIC", "-Wall", "-Wno-unused-function", "-I", str(CUDA / "include")]


def _sources():
    return sorted(p for p in CSRC.rglob("*") if p.suffix in (".cu", ".cpp"))


def _headers_stamp():
    h = hashlib.sha1()
    for p in sorted(list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list((ROOT / "include").rglob("*.h"))):
        h.update(str(p).encode())
        h.update(p.read_bytes())
    return h.hexdigest()[:12]


def build(force: bool = False, verbose: bool = False, jobs: int = 0) -> Path:
    BUILD.mkdir(exist_ok=True)
    stamp = _headers_stamp()
    objs, todo = [], []
    for src in _sources():
        h = hashlib.sha1(src.read_bytes() + stamp.encode()).hexdigest()[:12]
        obj = BUILD / f"{src.stem}.{h}.o"
        objs.append(obj)
        if obj.exists() and not force:
            continue
        if src.suffix == ".cu":
            cmd = [str(NVCC)] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)]
        todo.append((src, cmd))

    def compile_one(item):
        src, cmd = item
        if verbose:
            print(" ".join(cmd), flush=True)
        return src, subprocess.run(cmd, capture_output=True, text=True)

    # independent translation units: compiled concurrently (nvcc and g++ are separate processes)
    workers = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(compile_one, todo))
    for src, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"compile failed: {src.name}")
        if verbose and r.stderr.strip():
            sys.stderr.write(r.stderr)
    link = [str(NVCC)] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + [
        "-L", str(CUDA / "lib64"), "-lcudart", "-lz", "-Xlinker", "--no-undefined"]
    if verbose:
        print(" ".join(link), flush=True)
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    keep = set(objs)
    for old in BUILD.glob("*.o"):  # objects of earlier source versions
        if old not in keep:
            old.unlink()
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
