"""Build step of the CUDA library libhfgpu.so (sm_100a).

Regenerates the per-class kernels (csrc/gen_eri.py), compiles every
translation unit with nvcc in parallel into csrc/_build/, and links the
shared library next to this file.  Objects are rebuilt only when their
source or a shared header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libhfgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, deps) -> str:
    if not _newer(obj, [src] + deps):
        return ""
    cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = obj + ".log"
    with open(log, "w") as fh:
        fh.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-4000:]}")
    return src


def build(jobs: int = 0, verbose: bool = True) -> str:
    sys.path.insert(0, CSRC)
    try:
        import gen_eri  # noqa: E402
    finally:
        sys.path.pop(0)
    gen_srcs = gen_eri.main(os.path.join(CSRC, "generated"))
    os.makedirs(BUILD, exist_ok=True)
    common = [os.path.join(CSRC, "common.cuh"), os.path.join(CSRC, "types.cuh"), os.path.join(CSRC, "pairs.hpp"),
              os.path.join(CSRC, "scatter.cuh"),
              os.path.join(HERE, "..", "include", "hfgpu.h"),
              os.path.join(HERE, "..", "include", "hfgpu_basis.h"),
              os.path.join(HERE, "..", "include", "hfgpu_ingest.h"),
              os.path.join(HERE, "..", "include", "hfgpu_scf.h"),
              os.path.join(CSRC, "generated", "class_table.inc")]
    srcs = [os.path.join(CSRC, "hfgpu.cu"), os.path.join(CSRC, "onee.cu"), os.path.join(CSRC, "scf.cu"),
            os.path.join(CSRC, "ingest.cpp")] + sorted(gen_srcs)
    objs = [os.path.join(BUILD, os.path.splitext(os.path.basename(s))[0] + ".o") for s in srcs]
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, s, o, common + ([s[:-3] + ".cuh"] if os.path.exists(s[:-3] + ".cuh") else []))
                for s, o in zip(srcs, objs)]
        for f in futs:
            done = f.result()
            if done and verbose:
                print("compiled", os.path.basename(done), flush=True)
    if _newer(LIB, objs):
        # cuBLAS and cuSOLVER serve the device SCF step (scf.cu)
        subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
                              ["-lcublas", "-lcusolver", "-Xlinker", "-rpath=" + CUDA_LIB])
    return LIB


if __name__ == "__main__":
    build()
