"""Build recipe of the native library: nvcc for sm_100a, in-tree output.

``python -m cm_halofinder_b200.build`` compiles csrc/*.cu and csrc/*.cpp
into cm_halofinder_b200/libcmh_fof.so (CUDA runtime linked statically, so
the library does not depend on the runtime that other packages in the
process bring along).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcmh_fof.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def headers():
    out = [os.path.join(HERE, "..", "include", "cmh_fof.h")]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, jobs=8):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = headers()
    objs, cmds = [], []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if not _stale(obj, [src] + hdrs):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC, *ARCH, *CUFLAGS, "-c", src, "-o", obj]
        else:
            cmd = ["g++", *CXXFLAGS, "-I/usr/local/cuda/include", "-c", src, "-o", obj]
        cmds.append(cmd)
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT, text=True)))
        if len(procs) >= jobs:
            _wait(procs.pop(0), verbose)
    for p in procs:
        _wait(p, verbose)
    if cmds or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


def _wait(item, verbose):
    cmd, p = item
    out, _ = p.communicate()
    if p.returncode != 0:
        raise RuntimeError("compile failed: " + " ".join(cmd) + "\n" + out)
    if verbose and out.strip():
        print(out, flush=True)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
