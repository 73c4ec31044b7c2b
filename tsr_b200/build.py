"""Build the sm_100a core library in-tree (tsr_b200/lib/libtsrcore.so).

nvcc compiles every csrc/*.cu for sm_100a and links one shared library with
the C ABI of include/tsr_core.h.  The .so stays inside the package so that it
travels with the repository and is what every test and benchmark loads.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
OBJDIR = PKG / "lib" / "obj"
LIB = LIBDIR / "libtsrcore.so"
SOURCES = ["capi.cu", "tree.cu", "occupancy.cu", "dmc.cu", "mlp.cu", "noalloc.cu", "files.cu", "meshpost.cu", "depth.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", str(PKG.parent / "include")]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "tsr_core.h"]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJDIR.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    jobs = []
    for s in srcs:
        o = OBJDIR / (s.stem + ".o")
        if force or _stale(o, s):
            jobs.append([cc, *ARCH, *FLAGS, "-c", str(s), "-o", str(o)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [str(OBJDIR / (s.stem + ".o")) for s in srcs]
    if force or jobs or not LIB.exists():
        run([cc, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
