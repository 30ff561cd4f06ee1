"""Builds the sm_100a library and the care-b200 driver in place.

    python -m care_b200.build            # -> care_b200/libcareb200.so, care_b200/care-b200,
                                         #    care_b200/care-b200-peaks

Objects go to care_b200/_build/ (git-ignored). Every CUDA translation unit is
compiled for sm_100a only, with FMA contraction off (--fmad=false): the
correction path reproduces the reference's float arithmetic operation by
operation.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcareb200.so")
EXE = os.path.join(HERE, "care-b200")
PEAKS = os.path.join(HERE, "care-b200-peaks")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]

CU_SOURCES = ["capi.cu", "noalloc.cu", "mlp.cu", "tables.cu", "parse.cu"]
CXX_SOURCES = ["hostio.cpp", "readfile.cpp"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(HERE, "..", "include", "care_b200.h"))
    return out


def run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    objs, jobs = [], []
    for src in CU_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        if force or _newer(obj, deps):
            jobs.append([nvcc()] + NVFLAGS + ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        if force or _newer(obj, deps):
            jobs.append(["g++"] + CXXFLAGS + ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # translation units compile in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if force or _newer(LIB, objs):
        run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    if force or _newer(EXE, [LIB, os.path.join(CSRC, "main.cpp")]):
        run(["g++", "-O2", "-std=c++17", "-o", EXE, os.path.join(CSRC, "main.cpp"),
             "-L" + HERE, "-lcareb200", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    peaks_src = os.path.join(CSRC, "peaks.cu")
    if force or _newer(PEAKS, [peaks_src]):
        run([nvcc()] + ARCH + ["-O3", "-lineinfo", "-o", PEAKS, peaks_src])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
