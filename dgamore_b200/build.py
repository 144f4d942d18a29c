"""Builds the CUDA shared library ``libdga_b200.so`` in-tree for sm_100a (B200).

    python -m dgamore_b200.build            # compile (skips when up to date)
    python -m dgamore_b200.build --force

The library is plain CUDA C++ with an ``extern "C"`` ABI (see include/dga_b200.h); it links only the CUDA
runtime.  nvcc cross-compiles it without a GPU.
"""

from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_NAME = "libdga_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build dgamore_b200")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(
        glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h"))
    )


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(s) <= t for s in sources() + _headers())


def _compile_cmd(nvcc: str, src: str, obj: str, ptxas_info: bool) -> list[str]:
    cmd = [nvcc, *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-fmad=true", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(os.path.dirname(HERE), "include"), "-o", obj, src]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every .cu under csrc/ (one nvcc process per file, in parallel) and links them into one shared
    library next to this file; returns its path."""
    if not force and up_to_date():
        return LIB_PATH
    nvcc = nvcc_path()
    obj_dir = os.path.join(os.path.dirname(HERE), "_build", "obj")
    os.makedirs(obj_dir, exist_ok=True)
    jobs = []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = _compile_cmd(nvcc, src, obj, ptxas_info)
        if verbose:
            print(" ".join(cmd))
        jobs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    objs, errors = [], []
    for src, obj, proc in jobs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            errors.append(f"nvcc failed on {os.path.basename(src)} ({proc.returncode}):\n{out}\n{err}")
        elif ptxas_info or verbose:
            sys.stderr.write(err)
        objs.append(obj)
    if errors:
        raise RuntimeError("\n".join(errors))
    link = [nvcc, *ARCH_FLAGS, "-shared", "-Xcompiler", "-fPIC", "-o", LIB_PATH + ".tmp", *objs, "-lcudart"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose, ptxas_info=args.ptxas_info))


if __name__ == "__main__":
    main()
