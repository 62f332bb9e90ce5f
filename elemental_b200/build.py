"""Build recipe for libelemgpu.so (the sm_100a kernels + C ABI).

nvcc cross-compiles for sm_100a without a GPU.  The library is built in-tree
(elemental_b200/libelemgpu.so) so that it ships with the source tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libelemgpu.so")
BENCH_LIB = os.path.join(HERE, "libegpu_bench.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(BENCH_LIB):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(BENCH_LIB))
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(HERE, "bench_csrc", "*.cu")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compile every .cu in csrc/ for sm_100a and link libelemgpu.so."""
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                    "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            failed = True
            sys.stderr.write("FAILED: " + " ".join(cmd) + "\n")
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"],
                   check=True)
    os.replace(tmp, LIB)
    build_bench(flags)
    return LIB


def build_bench(flags: list[str]) -> str:
    """The benchmark-only library (bench_csrc/*.cu -> libegpu_bench.so): the
    FP64 peak probe that bench.py uses as its roofline denominator.  It is not
    linked into libelemgpu.so."""
    srcs = sorted(glob.glob(os.path.join(HERE, "bench_csrc", "*.cu")))
    tmp = BENCH_LIB + ".tmp"
    subprocess.run([nvcc()] + flags + ["-shared", "-o", tmp] + srcs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"],
                   check=True)
    os.replace(tmp, BENCH_LIB)
    return BENCH_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
