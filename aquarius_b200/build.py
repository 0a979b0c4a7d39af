"""Build recipe for libccsd_b200.so (in-tree, sm_100a).

python -m aquarius_b200.build   (or build() from __graft_entry__)
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "libccsd_b200.so"
BUILD = HERE / "_build"

CU = ["kernels_fp64.cu", "kernels_split.cu", "noalloc.cu"]
CPP = ["context.cpp", "planner.cpp", "solver.cpp", "hbuild.cpp", "fcidump.cpp", "capi.cpp", "synth.cpp", "split_exec.cpp",
       "server.cpp", "aomo.cpp", "plan_export.cpp", "diis.cpp", "merged.cpp"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + cmd[-1])
    return r


def _stale(src: Path, obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, jobs: int = 8) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + [ROOT / "include" / "ccsd_b200.h"]
    inc = ["-I" + str(ROOT / "include"), "-I" + str(CSRC)]
    cmds, objs = [], []
    for f in CU:
        src, obj = CSRC / f, BUILD / (f + ".o")
        objs.append(obj)
        if _stale(src, obj, headers):
            cmds.append([NVCC, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                         *inc, "-c", str(src), "-o", str(obj)])
    for f in CPP:
        src, obj = CSRC / f, BUILD / (f + ".o")
        objs.append(obj)
        if _stale(src, obj, headers):
            cmds.append(["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function",
                         "-I/usr/local/cuda/include", *inc, "-c", str(src), "-o", str(obj)])
    # compile in parallel
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c))
        procs.append((c, subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        if len(procs) >= jobs:
            c0, p0 = procs.pop(0)
            out, err = p0.communicate()
            if p0.returncode:
                raise RuntimeError("build step failed: " + " ".join(c0) + "\n" + out + err)
    for c0, p0 in procs:
        out, err = p0.communicate()
        if p0.returncode:
            raise RuntimeError("build step failed: " + " ".join(c0) + "\n" + out + err)
    if cmds or not OUT.exists():
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(OUT), *map(str, objs),
              "-L/usr/local/cuda/lib64", "-lcudart", "-lgomp"])
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
