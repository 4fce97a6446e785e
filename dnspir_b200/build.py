"""Builds the CUDA library (sm_100a) in-tree: dnspir_b200/libdnspir_b200.so.

Each source is compiled to an object in _build/ (in parallel), then the
objects are linked into the shared library."""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = ["api.cu", "fleet.cu", "encode.cu", "chain.cu", "scan.cu", "tscan.cu", "server.cu", "wire.cu", "client.cpp", "noalloc.cu"]
HEADERS = ["common.cuh", "ntt.cuh", "ntt2048.cuh", "kernels.cuh", "host.h", "fleet_impl.h"]
OUT = os.path.join(HERE, "libdnspir_b200.so")
OBJ_DIR = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"),
]


def build(verbose=False, extra=()):
    srcs = [os.path.join(HERE, "csrc", s) for s in SRC]
    deps = [os.path.join(HERE, "csrc", h) for h in HEADERS] + [os.path.join(ROOT, "include", "dnspir.h"),
                                                                os.path.abspath(__file__)]
    newest_dep = max(os.path.getmtime(p) for p in deps)
    if (os.path.exists(OUT) and os.path.getmtime(OUT) >= max(newest_dep, max(os.path.getmtime(p) for p in srcs))
            and not extra):
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        if (not extra and os.path.exists(obj) and
                os.path.getmtime(obj) >= max(newest_dep, os.path.getmtime(src))):
            return obj
        cmd = [NVCC, "-c", "-o", obj] + FLAGS + list(extra) + [src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [NVCC, "-shared", "-o", OUT, "-gencode", "arch=compute_100a,code=sm_100a"] + objs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
