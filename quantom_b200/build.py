"""Builds quantom_b200/liblima_b200.so in-tree with nvcc for sm_100a.

One shared library holds the C-ABI (include/lima_abi.h), the host engine
(C++) and the CUDA kernels.  Run ``python -m quantom_b200.build``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "liblima_b200.so"
BUILD = ROOT / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}", f"-I{CSRC}"]
# Reference-semantics kernels reproduce the reference's host-compiled float
# operation order: no a*b+c contraction into FMA in that translation unit.
PER_FILE = {"kernels_reference.cu": ["-fmad=false"], "nlist_reference.cu": ["-fmad=false"]}


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = Path(cuda) / "bin" / "nvcc"
    return str(p) if p.exists() else "nvcc"


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "lima_abi.h"]
    newest_hdr = max((h.stat().st_mtime for h in headers if h.exists()), default=0)
    objs = []
    nvcc = _nvcc()
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if not force and o.exists() and o.stat().st_mtime >= max(s.stat().st_mtime, newest_hdr):
            continue
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *PER_FILE.get(s.name, []), "-c", str(s), "-o", str(o)]
        if s.suffix == ".cpp":
            cmd = [nvcc, *NVCC_FLAGS, "-x", "cu", *ARCH, "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(OUT)
