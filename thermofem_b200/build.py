"""Builds libthermofem_b200.so (sm_100a) in-tree with nvcc.

    python -m thermofem_b200.build [--jobs N] [--verbose]

Every translation unit under thermofem_b200/csrc is compiled with
`-gencode arch=compute_100a,code=sm_100a -lineinfo -O3` into
thermofem_b200/_build/ and linked into thermofem_b200/lib/libthermofem_b200.so.
Objects are rebuilt when the source or any header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libthermofem_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++20", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                "--expt-relaxed-constexpr", "-ccbin", "g++",
                "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "**", "*.cu"), recursive=True))


def _headers():
    hs = glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    hs += glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
    # the C ABI header (the C++ component headers under include/ are not part of the library build)
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel[:-3] + ".o")


def _compile(src, verbose):
    obj = _obj(src)
    cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(jobs: int | None = None, verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _sources()
    newest_header = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    stale = [s for s in srcs if force or not os.path.exists(_obj(s))
             or os.path.getmtime(_obj(s)) < max(os.path.getmtime(s), newest_header)]
    failed = []
    if stale:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for src, rc, out in ex.map(lambda s: _compile(s, verbose), stale):
                if rc != 0:
                    failed.append((src, out))
                elif verbose and out.strip():
                    print(out)
    if failed:
        for src, out in failed:
            sys.stderr.write(f"--- {os.path.relpath(src, ROOT)}\n{out}\n")
        raise RuntimeError(f"nvcc failed for {len(failed)} translation unit(s)")
    objs = [_obj(s) for s in srcs]
    if stale or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    build_driver()
    return LIB


DRIVER_SRC = os.path.join(PKG, "driver", "solve_matrix.cpp")
DRIVER = os.path.join(PKG, "bin", "solve-matrix")


def build_driver() -> str:
    """The solve-matrix executable (host C++ over the C ABI, linked against
    the library with an rpath to thermofem_b200/lib)."""
    os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
    deps = [DRIVER_SRC, LIB] + glob.glob(os.path.join(ROOT, "include", "*.h"))
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(d) for d in deps):
        return DRIVER
    cmd = [NVCC, "-O2", "-std=c++20", "-ccbin", "g++", "-I", os.path.join(ROOT, "include"), DRIVER_SRC, "-o", DRIVER,
           "-L", LIBDIR, "-lthermofem_b200", "-Xlinker", "-rpath=$ORIGIN/../lib"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("solve-matrix build failed:\n" + r.stdout + r.stderr)
    return DRIVER


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose, a.force))
