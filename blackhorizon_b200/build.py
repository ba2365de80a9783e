"""Build libbh_b200.so in-tree with nvcc for sm_100a.

    python -m blackhorizon_b200.build [--verbose]

Compiles every .cu under blackhorizon_b200/csrc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and links one shared
library with the CUDA runtime linked statically, so the library only needs
the CUDA driver at run time.  ``-Xptxas -v`` output (registers, spills, shared
memory per kernel) is written to blackhorizon_b200/_build/ptxas.log.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbh_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put CUDA's bin on PATH")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "bh_b200.h"))
    return deps


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = False, defines=(), out: str = LIB) -> str:
    """Compile and link the library to `out`; `defines` are extra
    preprocessor definitions (NAME or NAME=VALUE)."""
    if not force and not defines and out == LIB and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    extra = [f"-D{d}" for d in defines]

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        cmd = [cc, *ARCH, *FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-c", src,
               "-o", obj]
        return obj, cmd, subprocess.run(cmd, capture_output=True, text=True)

    # The translation units are independent: compile them in parallel.
    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, sources()))
    objs = []
    log = []
    for obj, cmd, res in results:
        log.append(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed on {cmd[-3]}")
        objs.append(obj)
    tmp = out + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, out)
    with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("\n".join(log))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
