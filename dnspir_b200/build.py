"""Builds the CUDA library (sm_100a) in-tree: dnspir_b200/libdnspir_b200.so."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = ["api.cu", "fleet.cu", "encode.cu", "chain.cu", "scan.cu", "tscan.cu", "server.cu", "wire.cu", "client.cpp", "noalloc.cu"]
OUT = os.path.join(HERE, "libdnspir_b200.so")
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
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(HERE, "csrc", h) for h in
                                                   ("common.cuh", "ntt.cuh", "ntt2048.cuh", "kernels.cuh", "host.h", "fleet_impl.h")] +
                 [os.path.join(ROOT, "include", "dnspir.h")])
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= newest and not extra:
        return OUT
    cmd = [NVCC, "-shared", "-o", OUT] + FLAGS + list(extra) + srcs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
