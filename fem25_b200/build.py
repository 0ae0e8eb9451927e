"""Builds libfem25gpu.so in-tree for sm_100a (B200).

    python -m fem25_b200.build        # or fem25_b200.build.build()

nvcc cross-compiles without a GPU.  The plain-assembly and reference-
bookkeeping kernels are compiled with -fmad=false (no FMA contraction, the
reference's separately rounded arithmetic); everything else uses FMA.  The
plain element kernels are also compiled a second time with FMA allowed
(k_plain_fma.cu.o), the benchmark option of fem25_plain_fma.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfem25gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                 "-I", os.path.join(ROOT, "include"), "-I", SRC, "--expt-relaxed-constexpr"]

UNITS = [
    ("k_plain.cu", ["-fmad=false"]),
    ("k_plain.cu", ["-DFEM25_PLAIN_FMA"], "k_plain_fma.cu.o"),
    ("k_ref.cu", ["-fmad=false"]),
    ("k_batch.cu", []),
    ("k_grad.cu", []),
    ("k_grad_tc.cu", []),
    ("k_grad_cov.cu", []),
    ("api.cu", []),
    ("misfit_noalloc.cu", ["-fmad=false"]),
    ("dense_solve.cu", []),
    ("sparse_solve.cu", []),
]
HOST = [("host_setup.cpp", ["-O2", "-ffp-contract=off", "-fPIC", "-fopenmp", "-std=c++17"]),
        ("mesh_io.cpp", ["-O2", "-ffp-contract=off", "-fPIC", "-std=c++17"])]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "fem25gpu.h"))
    objs = []
    for unit in UNITS:
        name, flags = unit[0], unit[1]
        src = os.path.join(SRC, name)
        obj = os.path.join(OBJ, unit[2] if len(unit) > 2 else name + ".o")
        objs.append(obj)
        if _stale(obj, [src, __file__] + headers):
            out = _run([NVCC] + COMMON + list(flags) + list(extra) + ["-Xptxas", "-v", "-c", "-o", obj, src])
            if verbose:
                print(out)
    for name, flags in HOST:
        src = os.path.join(SRC, name)
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if _stale(obj, [src, __file__] + headers):
            _run(["g++"] + flags + ["-I", os.path.join(ROOT, "include"), "-I", SRC, "-c", "-o", obj, src])
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-lcusolver", "-lcublas"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
