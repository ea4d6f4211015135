"""Build libbd_aging_b200.so (sm_100a) and the drop-in CLI in-tree with nvcc.

    python -m bd_aging_b200.build          # or: python bd_aging_b200/build.py

Objects go to bd_aging_b200/_build/; the shared library and the CLI binary are
written next to this file so that they travel with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbd_aging_b200.so")
CLI = os.path.join(HERE, "bd_aging_self")

SOURCES = ["mirror.cu", "engine.cu", "correlate.cu", "gder.cu", "surrogate.cu", "cv3d.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"] + ARCH


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(ROOT, "include")
    return hs + [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    headers = _headers()
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _newer(o, [s] + headers) or ptxas_info:
            cmd = [nv] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(run, jobs):
            if verbose or ptxas_info:
                sys.stderr.write(out)
    if _newer(LIB, objs):
        run([nv] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    cli_src = os.path.join(CSRC, "cli", "bd_aging_self.cpp")
    if os.path.exists(cli_src) and _newer(CLI, [cli_src, LIB] + headers):
        run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), cli_src, "-o", CLI,
             "-L" + HERE, "-lbd_aging_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
