"""Build recipe of the CUDA library libhpq.so (sm_100a), in-tree next to this file."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhpq.so")
CLI = os.path.join(HERE, "hpq")
CLI_SRC = os.path.join(CSRC, "hpq_main.cpp")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def sources():
    out = []
    for root, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cuh", ".hpp", ".h")):
                out.append(os.path.join(root, f))
    out.append(os.path.join(os.path.dirname(HERE), "include", "hpq.h"))
    return out


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def cli_stale():
    if not os.path.exists(CLI):
        return True
    t = os.path.getmtime(CLI)
    return any(os.path.getmtime(s) > t for s in (CLI_SRC, LIB, os.path.join(os.path.dirname(HERE), "include", "hpq.h")))


def build(force=False, verbose=False):
    if force or needs_build():
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + NVCC_FLAGS + ["-o", tmp, os.path.join(CSRC, "api.cu"),
                                       os.path.join(CSRC, "poisson_noalloc.cu")]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    if force or cli_stale():
        build_cli(verbose)
    return LIB


def build_cli(verbose=False):
    """The command-line driver `hpq` (host C++ over the C ABI), linked against libhpq.so found
    next to it at run time."""
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-o", CLI, CLI_SRC, "-L" + HERE, "-lhpq",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)


if __name__ == "__main__":
    print(build(force=True, verbose=True))
