"""Builds libpfem2b.so in-tree for sm_100a with nvcc (no JIT, no torch).

Each translation unit is compiled to an object under _build/ in parallel
(the units share no device code), then nvcc links the shared library.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libpfem2b.so")
SOURCES = ["capi.cu", "particles.cu", "fem.cu", "krylov.cu", "amg.cu", "ale.cu", "project_noalloc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-fvisibility=hidden",
]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "pfem2.h")]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in _deps() if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    for s in SOURCES:
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        jobs.append((obj, [NVCC] + FLAGS + list(extra) + ["-c", os.path.join(CSRC, s), "-o", obj]))

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        list(ex.map(run, [c for _, c in jobs]))
    run([NVCC] + ARCH + ["-shared", "-cudart", "shared", "-o", OUT] + [o for o, _ in jobs])
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
