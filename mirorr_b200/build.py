"""Build recipe of the mirorr_b200 CUDA library (sm_100a only).

Compiles mirorr_b200/csrc/*.cu with nvcc into mirorr_b200/libmirorr_b200.so,
in tree, so the built library travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmirorr_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-DMIRORR_BUILD"]


def sources():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".cu"))


def _deps():
    files = sources() + [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".cuh")]
    files.append(os.path.join(HERE, "..", "include", "mirorr_b200.h"))
    return files


CLI_SRC = os.path.join(HERE, "cli")
CLI_OUT = os.path.join(HERE, "bin", "mirorr")
CXX = os.environ.get("CXX", "g++")


def build_cli(force: bool = False, verbose: bool = False) -> str:
    """The `mirorr` command line (mirorr_b200/cli) linked to the library."""
    srcs = sorted(os.path.join(CLI_SRC, f) for f in os.listdir(CLI_SRC) if f.endswith(".cpp"))
    deps = srcs + [os.path.join(CLI_SRC, f) for f in os.listdir(CLI_SRC) if f.endswith(".hpp")]
    deps += [OUT, os.path.join(SRC, "tfm.cuh")]
    if (not force and os.path.exists(CLI_OUT)
            and all(os.path.getmtime(f) <= os.path.getmtime(CLI_OUT) for f in deps)):
        return CLI_OUT
    os.makedirs(os.path.dirname(CLI_OUT), exist_ok=True)
    tmp = CLI_OUT + f".tmp{os.getpid()}"
    cmd = [CXX, "-O2", "-std=c++17", "-Wall", "-o", tmp, *srcs, f"-L{HERE}", "-lmirorr_b200",
           "-Wl,-rpath,$ORIGIN/..", "-lz"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, CLI_OUT)
    return CLI_OUT


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(sources()))) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = OUT + f".tmp{os.getpid()}"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC", "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
    print(OUT)
    print(build_cli(force="--force" in sys.argv, verbose=True))
