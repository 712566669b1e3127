"""Build libdjb200.so (sm_100a) in-tree with nvcc.

    python discodj.jl_b200/build.py [--force]

Compiles `csrc/*.cu` and `csrc/*.cpp` with `-gencode arch=compute_100a,code=sm_100a
-lineinfo -O3` into `discodj.jl_b200/lib/libdjb200.so`, linked against the
CUDA toolkit's cuFFT and cuBLAS (rpath to the toolkit's lib64). Rebuilds only when a source
or header is newer than the library unless --force is given.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libdjb200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) \
        + glob.glob(os.path.join(INCLUDE, "*.h")) + [os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = os.path.join(CUDA_HOME, "bin", "nvcc")
    common = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [*common, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    # one nvcc per translation unit, in parallel, then one link
    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, sources()))
    for obj, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({r.returncode}) on {obj}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)
    cmd = [nvcc, *ARCH, "--shared", *[o for o, _ in results], "-o", LIB + ".tmp",
           f"-L{CUDA_HOME}/lib64", "-lcufft", "-lcublas", "-Xlinker", f"-rpath,{CUDA_HOME}/lib64"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
