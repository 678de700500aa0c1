"""Builds the CUDA library ``libcavity_b200.so`` in-tree for sm_100a, and the
driver binary ``cavity_les`` (host C++ over the library's C ABI).

Each translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the FP64 units
(``prec_f64.cu``, ``oct_f64.cu``) additionally with ``-fmad=false`` so that its arithmetic
is that of the reference (no fused multiply-add) bit for bit.  The output
lands in ``cfd_cavity_b200/_build/``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libcavity_b200.so")
DRIVER = os.path.join(OUT, "cavity_les")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                 "-I" + os.path.join(HERE, "..", "include"), "--expt-relaxed-constexpr"]
UNITS = {
    "cavity.cu": [],
    "prec_f64.cu": ["-fmad=false"],
    "prec_f32.cu": [],
    "prec_f16.cu": [],
    "prec_bf16.cu": [],
    "prec_f16g.cu": [],
    "prec_f16sr.cu": [],
    "prec_bf16sr.cu": [],
    "prec_f16gsr.cu": [],
    "diag_noalloc.cu": [],
    "octree_api.cu": [],
    "oct_f64.cu": ["-fmad=false"],
    "oct_f32.cu": [],
    "oct_f16.cu": [],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> str:
    os.makedirs(OUT, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "cavity.h"))
    objs = []
    jobs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OUT, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _sources_newer(obj, [src, __file__] + headers):
            jobs.append([nvcc(), *COMMON, *flags, *extra_flags, "-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if jobs or not os.path.exists(LIB):
        run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    drv_src = [os.path.join(CSRC, "driver.cpp"), os.path.join(CSRC, "rustfmt.h"),
               os.path.join(HERE, "..", "include", "cavity.h")]
    if force or _sources_newer(DRIVER, drv_src + [LIB, __file__]):
        run([shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall", "-Wextra",
             "-I" + os.path.join(HERE, "..", "include"), "-I" + CSRC, drv_src[0], "-o", DRIVER,
             "-L" + OUT, "-lcavity_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
