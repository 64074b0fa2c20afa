"""In-tree build of the native libraries.

* ``liblare_gpu.so``  - sm_100a CUDA engine + C ABI (include/lare_gpu.h) and
  the learned-conduction kernels (include/lare_surrogate.h)
* ``liblare_host.so`` - host helpers of the deck layer (KISS generator)

Run ``python -m lare3d_b200.build``.  Object files go to ``_build/`` and the
shared libraries next to this file, so they travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = [
    "-std=c++17", "-O3", "-lineinfo", "--extended-lambda", "-Xcompiler", "-fPIC",
    "-Werror", "cross-execution-space-call", "-diag-suppress", "20011",
]

# (source, extra flags).  The exact FP64 engine rounds every operation
# separately (--fmad=false) to reproduce the reference's x86-64 arithmetic bit
# for bit; the product FP64 engine contracts multiply-adds.
UNITS = [
    ("engine_f64fast.cu", ["--fmad=true"]),
    ("engine_f64.cu", ["--fmad=false"]),
    ("engine_f32.cu", ["--fmad=true", "-prec-div=false", "-prec-sqrt=false"]),
    ("lare_gpu.cu", []),
    ("lare_noalloc.cu", ["--fmad=false"]),
    ("surrogate.cu", []),
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = [os.path.join(ROOT, "include", h) for h in ("lare_gpu.h", "lare_surrogate.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".h", ".cu")):
            out.append(os.path.join(CSRC, f))
    return out


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    deps = _deps()
    so = os.path.join(HERE, "liblare_gpu.so")

    def compile_unit(unit):
        src, extra = unit
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        if not force and not _newer(obj, deps):
            return obj, ""
        cmd = [cc, *NVCC_COMMON, *ARCH, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        results = list(ex.map(compile_unit, UNITS))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    if force or _newer(so, objs):
        cmd = [cc, "-shared", *ARCH, "-o", so, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    host_so = os.path.join(HERE, "liblare_host.so")
    host_src = os.path.join(CSRC, "lare_host.c")
    if force or _newer(host_so, [host_src]):
        r = subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-o", host_so, host_src], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host helper build failed:\n{r.stderr}")
    return so


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv))
