"""Build libcbf.so in-tree: every CUDA source compiled for sm_100a with nvcc.

    python cudabifurcation3.0_b200/build.py [--force] [--verbose]

Objects go to cudabifurcation3.0_b200/_build/, the library to
cudabifurcation3.0_b200/libcbf.so (both git-ignored; the .so travels with the
source tree).  -fmad=false: the only fused multiply-adds are the explicit fma()
calls of the model steps, which the CPU oracle evaluates identically.
"""
from __future__ import annotations

import argparse
import os
import shutil
from concurrent.futures import ThreadPoolExecutor
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcbf.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fvisibility=default",
    "-diag-suppress", "177,550",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = headers()
    objs, cmds = [], []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or ptxas_info or _stale(obj, [src, *hdrs]):
            cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_info and src.suffix == ".cu":
                cmd.insert(1, "-Xptxas=-v")
            if src.suffix == ".cpp":
                cmd[1:1] = ["-x", "cu"]
            if verbose:
                print(" ".join(cmd), flush=True)
            cmds.append(cmd)
    # translation units are independent: compile them concurrently
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=ptxas_info, text=True), cmds):
            if ptxas_info:
                sys.stdout.write(r.stdout)
                sys.stderr.write(r.stderr)
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args(argv)
    path = build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
