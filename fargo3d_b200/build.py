"""Build libfargo_b200.so in-tree (nvcc for sm_100a + gcc for the C host side).

    python -m fargo3d_b200.build

The FP64 kernels are compiled with --fmad=false so that their arithmetic
rounds exactly as the reference's CPU build; the FP32 kernels keep FMA.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
BUILD = os.path.join(ROOT, "_build", "fargo3d_b200")
LIB = os.path.join(OUT, "libfargo_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".c", ".cuh", ".h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return all(os.path.getmtime(s) <= t for s in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    fast32 = [] if os.environ.get("FB_FP32_IEEE") else ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
    cu_flags = {"fb_kernels_f64.cu": ["--fmad=false"], "fb_kernels_f32.cu": fast32, "fb_noalloc.cu": ["--fmad=false"],
                "fb_batch_f64.cu": ["--fmad=false"], "fb_batch_f32.cu": fast32}
    cmds = []
    for f in sorted(os.listdir(CSRC)):
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if f.endswith(".cu"):
            cmd = [nvcc] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-Xptxas", "-v"] + cu_flags.get(f, []) + INC + ["-c", src, "-o", obj]
        elif f.endswith(".c"):
            cmd = ["gcc", "-O2", "-std=gnu99", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                   "-I/usr/local/cuda/include"] + INC + ["-c", src, "-o", obj]
        else:
            continue
        cmds.append(cmd)
        objs.append(obj)
    # translation units are independent: compile them concurrently
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for out in ex.map(_run, cmds):
            if verbose:
                sys.stdout.write(out)
    _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lm", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
