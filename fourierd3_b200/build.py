"""Build libfd3.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

    python -m fourierd3_b200.build        # or: python fourierd3_b200/build.py

nvcc compiles every .cu under csrc/ for ``-gencode arch=compute_100a,code=sm_100a``
and links cuFFT; the result is fourierd3_b200/_lib/libfd3.so.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfd3.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "--extended-lambda",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(os.path.dirname(HERE), "include", "fd3.h"))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    jobs = []
    for src in sources():
        obj = os.path.join(OUT_DIR, os.path.basename(src)[:-3] + ".o")
        jobs.append(([NVCC, *FLAGS, *extra, "-c", src, "-o", obj], obj))
    if verbose:
        for cmd, _ in jobs:
            print(" ".join(cmd))
    workers = min(len(jobs), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(workers) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[0], capture_output=True, text=True), jobs))
    failed = [r for r in results if r.returncode != 0]
    for r in results:
        if r.stderr and (verbose or r.returncode != 0):
            sys.stderr.write(r.stderr)
    if failed:
        raise RuntimeError(f"nvcc failed for {len(failed)} source file(s)")
    objs = [o for _, o in jobs]
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
           "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
           "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


TORCH_SRC = os.path.join(HERE, "csrc_torch", "fd3_torch_ops.cpp")
TORCH_LIB = os.path.join(OUT_DIR, "libfd3_torch.so")


def build_torch_ops(force: bool = False, verbose: bool = False) -> str:
    """The thin torch operator library (torch.ops.fd3.*) over the C ABI: g++ against the
    installed torch headers and libraries, linked to libfd3.so (found next to it at run time)."""
    import torch

    deps = [TORCH_SRC, LIB, os.path.join(os.path.dirname(HERE), "include", "fd3.h")]
    if (not force and os.path.exists(TORCH_LIB)
            and all(os.path.getmtime(d) <= os.path.getmtime(TORCH_LIB) for d in deps)):
        return TORCH_LIB
    tdir = os.path.dirname(torch.__file__)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-I" + os.path.join(tdir, "include"), "-I" + os.path.join(tdir, "include", "torch", "csrc", "api", "include"),
           "-I" + os.path.join(CUDA_HOME, "include"), "-I" + os.path.join(os.path.dirname(HERE), "include"),
           TORCH_SRC, "-o", TORCH_LIB + ".tmp",
           "-L" + OUT_DIR, "-lfd3", "-L" + os.path.join(tdir, "lib"), "-ltorch", "-ltorch_cpu", "-ltorch_cuda",
           "-lc10", "-lc10_cuda", "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(tdir, "lib")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(TORCH_LIB + ".tmp", TORCH_LIB)
    return TORCH_LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(force=True, verbose=True, extra=extra))
